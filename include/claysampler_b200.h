/*
 * claysampler_b200 — C ABI of the B200 batch voice renderer.
 *
 * The renderer is a drop-in for ClaySampler's device half: the planner hands it
 * one `cs_plan` per job (the reference's `clay::RenderPlan`, src/render/plan.h:9-20)
 * and it returns PCM16 plus one `cs_tail_result` per job (the reference's
 * `clay::RenderBatch`, src/cuda/renderer.h:37-43).  All entry points return 0 on
 * success and a nonzero status on failure; `cs_last_error` gives the message
 * (the reference throws std::runtime_error from Driver::check,
 * src/cuda/renderer.cpp:69-77, which its CLI turns into `ERROR\t...`, exit 1).
 *
 * The POD records below are byte-compatible with the reference's shared host/device
 * structs in src/cuda/render_types.h, so a planner built against either header can
 * pass its arrays through unchanged.  Field names follow the reference.
 */
#ifndef CLAYSAMPLER_B200_H
#define CLAYSAMPLER_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- enumerations (src/cuda/render_types.h:3-15, 105-108) ---------------------- */
enum cs_mod_target {
    CS_MOD_AMPLITUDE, CS_MOD_VOLUME, CS_MOD_PAN, CS_MOD_WIDTH, CS_MOD_POSITION, CS_MOD_PITCH,
    CS_MOD_ENV_DELAY, CS_MOD_ENV_ATTACK, CS_MOD_ENV_HOLD, CS_MOD_ENV_DECAY, CS_MOD_ENV_SUSTAIN,
    CS_MOD_ENV_START, CS_MOD_ENV_RELEASE, CS_MOD_OFFSET, CS_MOD_DELAY,
    CS_MOD_CUTOFF, CS_MOD_RESONANCE, CS_MOD_CUTOFF2, CS_MOD_RESONANCE2,
    CS_MOD_FILTER_VELOCITY, CS_MOD_FILTER_VELOCITY2,
    CS_MOD_LFO_FREQUENCY, CS_MOD_LFO_PHASE, CS_MOD_LFO_DELAY, CS_MOD_LFO_FADE,
    CS_MOD_FILEG_DELAY, CS_MOD_FILEG_ATTACK, CS_MOD_FILEG_HOLD, CS_MOD_FILEG_DECAY,
    CS_MOD_FILEG_SUSTAIN, CS_MOD_FILEG_START, CS_MOD_FILEG_RELEASE,
    CS_MOD_PITCHEG_DELAY, CS_MOD_PITCHEG_ATTACK, CS_MOD_PITCHEG_HOLD, CS_MOD_PITCHEG_DECAY,
    CS_MOD_PITCHEG_SUSTAIN, CS_MOD_PITCHEG_START, CS_MOD_PITCHEG_RELEASE,
    CS_MOD_FILEG_DEPTH, CS_MOD_PITCHEG_DEPTH,
    CS_MOD_EQ1_FREQUENCY, CS_MOD_EQ1_BANDWIDTH, CS_MOD_EQ1_GAIN,
    CS_MOD_EQ2_FREQUENCY, CS_MOD_EQ2_BANDWIDTH, CS_MOD_EQ2_GAIN,
    CS_MOD_EQ3_FREQUENCY, CS_MOD_EQ3_BANDWIDTH, CS_MOD_EQ3_GAIN
};

enum cs_filter_type {
    CS_FILTER_NONE, CS_FILTER_LOW1, CS_FILTER_HIGH1, CS_FILTER_LOW2, CS_FILTER_HIGH2,
    CS_FILTER_BAND2, CS_FILTER_NOTCH2, CS_FILTER_LOW4, CS_FILTER_HIGH4, CS_FILTER_BAND4,
    CS_FILTER_LOW6, CS_FILTER_HIGH6, CS_FILTER_BAND6, CS_FILTER_PEAK
};

enum cs_generator { CS_GEN_NONE, CS_GEN_SINE, CS_GEN_SILENCE, CS_GEN_NOISE };

enum cs_tail_status {
    CS_TAIL_OK, CS_TAIL_DURATION, CS_TAIL_NONFINITE, CS_TAIL_PEAK, CS_TAIL_AUDIO_DURATION,
    CS_TAIL_QUIET_PERFORMANCE, CS_TAIL_EXCESSIVE_SILENCE, CS_TAIL_SILENT_AUDIO, CS_TAIL_CLIPPING,
    CS_TAIL_SILENT_BODY, CS_TAIL_INCOMPLETE_GROUP, CS_TAIL_SCRATCH_MEMORY
};

#define CS_FILTER_SLOTS 5
#define CS_TAIL_BLOCK_FRAMES 1024      /* src/cuda/render_types.h:92 */
#define CS_NATURAL_TAIL_LIMIT_SECONDS 120

/* ---- plan records (src/cuda/render_types.h:30-90) -------------------------------- */
typedef struct cs_voice_filter {
    int32_t type;                        /* enum cs_filter_type */
    float cutoff, resonance, bandwidth, gain;
} cs_voice_filter;

typedef struct cs_envelope_shape {
    int32_t attackStart, holdStart, decayStart, releaseStart, fadeStart;
    float start, attackStep, decayRate, sustain, releaseValue, releaseRate, fadeValue, fadeStep;
    float depth, releaseSeconds;
} cs_envelope_shape;

/* One contiguous span of one voice (src/cuda/render_types.h:41-68), 472 bytes. */
typedef struct cs_voice_span {
    uint64_t sample;                     /* offset of frame 0 in the float bank */
    double position, step, pitchSlope;
    int32_t channels, begin, end, sourceEnd, loopFirst, loopEnd, loopCrossfade;
    int32_t stereoMatrix;
    int32_t generator;                   /* enum cs_generator */
    uint32_t noiseSeed;
    int32_t noiseStart;
    int32_t firstModulation, modulationCount;
    int32_t firstLfo, lfoCount;
    int32_t filterTrack, nextFilteredSpan;
    uint64_t filteredOffset, phaseOffset;
    int32_t variablePitch;
    float minimumPitchRatio;
    int32_t filterControls[4];
    int32_t sampleRate;
    cs_voice_filter filters[CS_FILTER_SLOTS];
    cs_envelope_shape extraEnvelope[2];
    int32_t activeEnvelope[2];
    int32_t attackStart, holdStart, decayStart, releaseStart, fadeStart, bendEnd;
    float gain, pan, left, right, start, attackStep, decayRate, sustain, releaseValue, releaseRate;
    float fadeValue, fadeStep;
    float widthDirect, widthCross, positionLeft, positionRight;
    float width, stereoPosition;
} cs_voice_span;

/* Piecewise-linear control track point (src/cuda/render_types.h:76-79). */
typedef struct cs_control_point {
    int32_t frame;
    float value, step;
} cs_control_point;

/* Modulation binding (src/cuda/render_types.h:81-86).  In a plan, `first` and
 * `shapeFirst` are track indices (or -1); the renderer rebases them to points. */
typedef struct cs_voice_modulation {
    int32_t first, last;
    int32_t target;                      /* enum cs_mod_target */
    float depth;
    int32_t shapeFirst, shapeLast;
} cs_voice_modulation;

/* Quality-gate configuration (src/cuda/render_types.h:110-114). */
typedef struct cs_audio_config {
    int32_t rate, window, maxFrames, minPeak;
    uint8_t enabled;
    double minMedian, minQuartile, silencePower, maxSilentFraction, maxSilentFrames, maxClippedFraction;
} cs_audio_config;

typedef struct cs_audio_metrics {
    double median, quartile, silentFraction, clippedFraction, bodyRms, targetRms, gain;
    int32_t longestSilence, clipped;
    int32_t verdict;                     /* enum cs_tail_status */
    uint8_t measured;
} cs_audio_metrics;

/* Per-job result (src/cuda/render_types.h:134-140), 112 bytes. */
typedef struct cs_tail_result {
    uint64_t offset;                     /* first frame of this job in the batch PCM */
    int32_t frames, dataFrames, fade, peak, first, last;
    int32_t status;                      /* enum cs_tail_status */
    float scale;
    cs_audio_metrics audio;
} cs_tail_result;

/* One render job (clay::RenderPlan, src/render/plan.h:9-20) as flat arrays.
 * Control track i is points[track_offsets[i] .. track_offsets[i+1]).  Tracks 0..2
 * are the job's CC7, CC11 and CC10 automation (src/render/plan.cpp:296-305). */
typedef struct cs_plan {
    const cs_voice_span* spans;
    const cs_control_point* points;
    const int64_t* track_offsets;        /* track_count + 1 entries */
    const cs_voice_modulation* modulation;
    const int32_t* onsets;
    int32_t span_count, track_count, modulation_count, onset_count;
    int32_t filter_tracks, frames, music_end, limit, fade_frames, tail_clipped, body_frames;
    uint64_t volume_group;
} cs_plan;

/* ---- renderer (clay::Renderer, src/cuda/renderer.h:45-64) ---------------------- */
typedef struct cs_renderer cs_renderer;

/* A finished batch (clay::RenderBatch).  `pcm` holds result.dataFrames frames per
 * accepted job starting at result.offset, mono in natural mode and interleaved
 * stereo otherwise; it stays valid only during the publish callback. */
typedef struct cs_batch {
    const int16_t* pcm;
    size_t pcm_samples;
    const cs_tail_result* results;
    size_t result_count;
    double kernel_seconds;
    size_t failed_scratch_bytes;         /* single rejected job at `first` */
    const size_t* job_indices;           /* noncontiguous completions, else NULL */
    size_t job_index_count;
} cs_batch;

typedef void (*cs_publish_fn)(void* user, const cs_batch* batch, size_t first);
/* Appends more plans while rendering (clay::Renderer::Refill).  Returns 1 and sets
 * `plans`/`count` to an array that stays valid until the renderer publishes those
 * jobs, or returns 0 when nothing is ready (`wait` = 0) or no work remains. */
typedef int (*cs_refill_fn)(void* user, int wait, const cs_plan** plans, size_t* count);

/* Replaces Renderer::Renderer (src/cuda/renderer.h:47-48, renderer.cpp:491-546).
 * `natural` selects the float mix with natural-tail finishing (mono PCM16);
 * otherwise the mix is stereo PCM16 (orig/custom).  No NVRTC path: the kernels are
 * compiled offline for sm_100a. */
int cs_renderer_create(int device, int natural, const cs_audio_config* audio, int group_minimum,
                       size_t waiting_limit, size_t batch_jobs, cs_renderer** out);
void cs_renderer_destroy(cs_renderer* renderer);

/* Replaces Renderer::uploadSamples (src/cuda/renderer.cpp:553-603): the bank is
 * interleaved float32; only the tail beyond the last upload is copied unless
 * `fresh` restarts the bank. */
int cs_upload_samples(cs_renderer* renderer, const float* pcm, size_t floats, int fresh);

/* Replaces Renderer::renderWindow (src/cuda/renderer.cpp:1748-1820): renders every
 * plan and calls `publish` once per finished batch with the index of its first job. */
int cs_render_window(cs_renderer* renderer, const cs_plan* plans, size_t count,
                     cs_publish_fn publish, cs_refill_fn refill, void* user);

/* ---- serving: non-blocking submission (no reference counterpart) ---------------
 * Continuous batching for a render service: cs_submit queues plans and returns at
 * once, after staging and launching what the renderer's free stream lanes take
 * (two batches in flight, each up to batch_jobs plans; volume-group rules as in
 * cs_render_window).  cs_poll publishes finished batches in order through
 * `publish` (whose `first` is the ticket of the batch's first job) and admits queued
 * plans into the lanes that freed up; with `wait` it blocks for the oldest batch
 * in flight.  Tickets number submitted plans from 0 in submission order.  A
 * plan's arrays must stay valid until its job is published.  cs_render_window
 * refuses to run while submitted jobs are unpublished. */
int cs_submit(cs_renderer* renderer, const cs_plan* plans, size_t count, uint64_t* first_ticket);
int cs_poll(cs_renderer* renderer, int wait, cs_publish_fn publish, void* user, size_t* published);
/* Submitted jobs not yet published (queued or in flight). */
size_t cs_pending_jobs(const cs_renderer* renderer);

/* Getters (src/cuda/renderer.h:54-59). */
const char* cs_renderer_device(const cs_renderer* renderer);
size_t cs_peak_bytes(const cs_renderer* renderer);
size_t cs_sample_cache_budget(const cs_renderer* renderer);
size_t cs_peak_waiting_bytes(const cs_renderer* renderer);
size_t cs_spilled_bytes(const cs_renderer* renderer);
size_t cs_downloaded_bytes(const cs_renderer* renderer);

/* Message of the last failed call on this thread (no reference counterpart: the
 * reference reports failures as C++ exceptions). */
/* The message of the last failed call on this renderer (empty when none): the
 * reference's exception text for that renderer, where cs_last_error is the calling
 * thread's. */
const char* cs_renderer_last_error(const cs_renderer* renderer);
const char* cs_last_error(void);

/* ---- staged batches (measurement and tests; no reference counterpart) -----------
 * A prepared batch keeps its plans' device metadata, mix and finishing buffers
 * resident so that the synthesis + finishing pass can be re-run on device-resident
 * inputs, the boundary at which kernel throughput is measured. */
typedef struct cs_prepared cs_prepared;

int cs_prepare(cs_renderer* renderer, const cs_plan* plans, size_t count, cs_prepared** out);
/* Enqueues synthesis and finishing on `stream` (a cudaStream_t, NULL = the
 * renderer's stream); does not synchronise. */
int cs_run(cs_renderer* renderer, cs_prepared* batch, void* stream);
/* Synchronises and copies results; `pcm` may be NULL to query `*pcm_samples`. */
int cs_collect(cs_renderer* renderer, cs_prepared* batch, int16_t* pcm, size_t pcm_capacity,
               size_t* pcm_samples, cs_tail_result* results);
/* Copies the synthesised mix (float2 per frame in natural mode, short2 otherwise)
 * for all jobs, concatenated in plan order. */
int cs_copy_mix(cs_renderer* renderer, cs_prepared* batch, void* host, size_t bytes);
size_t cs_prepared_frames(const cs_prepared* batch);
/* Device address and size of that mix, valid until the batch is destroyed or run
 * again; the caller orders its reads after cs_run's work (same stream, or an event). */
int cs_prepared_mix_device(const cs_prepared* batch, const void** mix, size_t* bytes);
/* Kernel launches the last cs_run enqueued. */
int cs_prepared_launches(const cs_prepared* batch);
void cs_prepared_destroy(cs_prepared* batch);
/* Per-stage device timing of the next cs_run calls (events between stages). */
int cs_prepared_set_profile(cs_prepared* batch, int enable);
/* Fills ms[stage] (stages: 0 pitch, 1 source, 2 recurrence, 3 general chains,
 * 4 mix + block scan, 5 finishing) for the last profiled run; returns the stage
 * count or -1. */
int cs_prepared_stage_ms(cs_prepared* batch, float* ms, int capacity);
const char* cs_stage_name(int stage);

/* Number of synthesis segments the batch was cut into. */
size_t cs_prepared_segments(const cs_prepared* batch);

/* Caps the chain-storage bytes of one synthesis segment (0 = derive the budget
 * from free device memory).  No reference counterpart: the reference exercises
 * segmentation with a special build that limits scratch to 64 KiB
 * (docs/validation.md:145). */
int cs_renderer_set_scratch_limit(cs_renderer* renderer, size_t bytes);

/* Shared voice sources (on by default).  No counterpart in the reference, whose
 * renderTiles / renderFilterSources resample every voice frame (src/cuda/render.cu:
 * 138-215).  Voices without a filter chain that play the same sample from the same
 * position at the same step, with the same loop, loop crossfade and pitch ramp,
 * have the same resampled source at every elapsed frame; with this on, a batch
 * renders each such source once (48-tap sinc, loop wrap and crossfade) and the
 * mix reads it for every voice that plays it.  The audio is identical either way
 * (the same arithmetic on the same values); off is the plain path, which
 * resamples every voice frame inline.  Applies to batches prepared afterwards. */
int cs_renderer_set_shared_sources(cs_renderer* renderer, int enable);
/* Host milliseconds the renderer spent staging batches so far, per phase: batch
 * index (voices, tiles, jobs), scratch budget, segment plan, shared-source plan,
 * arena, staging pieces, staging copies and upload issue, upload wait; then two
 * device times of the batches render_window / cs_poll published: their download
 * copies and their kernels.  Writes up to `capacity` values and returns the count.
 * No counterpart in the reference. */
int cs_renderer_host_ms(const cs_renderer* renderer, double* ms, int capacity);
/* Batches in flight at most (1-4, default 2), each on its own stream lane with its
 * own arena.  cs_render_window publishes batches in order; cs_poll publishes them
 * as they finish.  The reference keeps one rolling batch of resident jobs
 * (src/cuda/renderer.cpp:1353-1746). */
int cs_renderer_set_lanes(cs_renderer* renderer, int lanes);
/* Host-side fault injection for tests: the next `count` batch-arena allocations
 * report cudaErrorMemoryAllocation without calling the allocator, so the
 * out-of-memory ladder of cs_render_window / cs_poll runs (publish the batches in
 * flight and free the other lanes' arenas, halve the batch, halve a lone job's
 * scratch budget, reject the job; src/cuda/renderer.cpp:947-992).  0 turns it off. */
int cs_renderer_fail_allocations(cs_renderer* renderer, int count);
/* 1 (default): render windows and serving run every lane's kernels on one stream
 * in batch order (the oldest batch finishes first and its download overlaps the
 * next batches' kernels), and a render window pools its shared voice sources
 * across its batches.  0: each lane runs its kernels on its own stream beside the
 * others, which suits batches whose latency-bound kernels (long filter chains)
 * leave the GPU room, and shared sources are planned per batch.  The audio is the
 * same either way.  No counterpart in the reference. */
int cs_renderer_set_ordered_compute(cs_renderer* renderer, int ordered);
/* Serving: how often a batch launch waited because its estimated footprint
 * exceeded half of the free device memory while other batches were in flight. */
size_t cs_renderer_deferred_launches(const cs_renderer* renderer);
/* Shared sources of a prepared batch, the floats they hold, and the voice frames
 * that read them instead of resampling. */
size_t cs_prepared_shared_sources(const cs_prepared* prepared);
size_t cs_prepared_shared_frames(const cs_prepared* prepared);
long long cs_prepared_shared_voice_frames(const cs_prepared* prepared);
/* Channel-frames of the shared sources that run the 48-tap sinc (step or pitch
 * ramp away from 1); `voice_floats` receives those of the voices reading them,
 * which the mix no longer resamples. */
long long cs_prepared_shared_sinc(const cs_prepared* prepared, long long* voice_floats);

/* ---- natural-tail finishing without device allocation --------------------------
 * No counterpart in the reference (its finishing always runs inside the renderer
 * on renderer-owned scratch).  For callers that cannot allocate device memory
 * while they render: a real-time audio host calling in from its audio callback,
 * where cudaMalloc can block or synchronise the device past the callback's
 * deadline, or an application embedding the renderer that owns the device-memory
 * budget itself.  The caller passes the float mix (float2 per frame, jobs
 * concatenated in order) and the outputs, all in device memory; the stage's
 * intermediates live in a fixed file-scope device array of about 17 MiB that every
 * GPU loading the library holds until exit.  Limits per call:
 * CS_STATIC_FINISH_MAX_FRAMES frames and CS_STATIC_FINISH_MAX_JOBS jobs (larger
 * calls fail with a message from cs_finish_natural_static_error); window >= 400.
 * The first call on each device looks up the array's device address with that
 * device current; with CUDA's lazy module loading (the default) that first
 * lookup also loads the library's device code and places the array, which can
 * allocate and synchronise, so make the first call at set-up time, outside the
 * real-time path and before any stream capture.  Later calls allocate nothing:
 * the job records travel to the device inside a set-up kernel's launch
 * parameters (no pageable host-to-device copy).  All calls share the array:
 * calls whose work overlaps on the GPU race and must be serialised.
 * `packed` receives up to the sum of frames int16 samples and `results` one
 * cs_tail_result per job, exactly as the renderer's natural finishing writes
 * them.  Enqueued on `stream` (a cudaStream_t; NULL = the legacy default stream);
 * returns 0 once enqueued. */
#define CS_STATIC_FINISH_MAX_FRAMES (1u << 23)
#define CS_STATIC_FINISH_MAX_JOBS 256

typedef struct cs_finish_job {
    int32_t frames, music_end, limit, fade_frames;
} cs_finish_job;

int cs_finish_natural_static(const float* mix, const cs_finish_job* jobs, int count, int rate, int window,
                             int16_t* packed, cs_tail_result* results, void* stream);
const char* cs_finish_natural_static_error(void);

#ifdef __cplusplus
}
#endif

#endif
