// Device records and kernel launchers shared by the renderer's host code.
#pragma once

#include "../../include/claysampler_b200.h"
#include <cuda_runtime.h>
#include <stdint.h>

namespace cs {

constexpr int kTaps = 48;               // render.cu:3
constexpr int kPhases = 2048;           // render.cu:4
constexpr int kTileFrames = 256;       // frames per mix tile (one voice list each)
constexpr int kBlockFrames = CS_TAIL_BLOCK_FRAMES;
constexpr int kTilesPerBlock = kBlockFrames / kTileFrames;
constexpr int kSourceTile = 256;         // frames per source-kernel CTA
#ifndef CS_SOURCE_THREADS
#define CS_SOURCE_THREADS 128
#endif
constexpr int kSourceThreads = CS_SOURCE_THREADS;   // threads per source-kernel CTA
static_assert(kSourceTile % kSourceThreads == 0, "whole frames per source thread");
constexpr uint64_t kNoTargets = ~uint64_t(0);
constexpr int kRecChainsPerCta = 32;     // single-slot chains per recurrence CTA
#ifndef CS_LEAD_TIERS
#define CS_LEAD_TIERS 3
#endif
constexpr int kLeadTiers = CS_LEAD_TIERS; // tiers of long chains whose recurrences start early
// Moving-filter targets are stored per 32-frame chunk as three planes
// (c0[32], c1[32], c2[32]) so the recurrence reads four frames per 128-bit load.
constexpr int kRecChunkFrames = 32;
// Host phases of staging a batch, timed per renderer: index building, scratch
// budget, segment planning, shared-source planning, arena, staging pieces,
// staging copies and upload issue, upload wait.
constexpr int kHostPhases = 10;
// The last two entries of the staging-time counters are device times of the
// published batches: their download copies and their kernels.
constexpr int kPhaseDownload = 8, kPhaseKernels = 9;

// A mix tile: kTileFrames frames of one job with the spans that overlap it
// (the reference's Tile, src/cuda/render_types.h:70-74).
struct MixTile {
    int first, count;                   // range in the voice index list
};

// A job's spans in the batch and where its tile voice lists start in the batch's
// index list (tileIndexKernel builds the lists on the device).
struct JobSpans {
    int voiceFirst, voiceCount, indexFirst, unused;
};

// Tiles of a job that one tileIndexKernel CTA lists.
constexpr int kIndexChunkTiles = 2048;

struct JobInfo {
    uint64_t offset;                    // first frame of the job in the batch mix
    int frames, musicEnd, limit, fade;
    int blockFirst, windowFirst, tileFirst;
    int tracks[4];                      // point offsets bounding CC7, CC11, CC10
};

// Recurrence state of one voice chain carried across segments
// (the reference's VoiceState, src/cuda/render_types.h:22-28).
struct ChainState {
    double position, step;
    int pitchSpan, previousLoopEnd, previousLoopStart;
    int pitchInitialized, filterInitialized;
    int pad;
    float z1[CS_FILTER_SLOTS][3][2], z2[CS_FILTER_SLOTS][3][2];
    float coefficients[CS_FILTER_SLOTS][5];
};

struct StereoStats { double power; float peak; };
struct MonoStats { double power; int peak; };

struct TailConfig {                     // src/cuda/render_types.h:100-103
    int window, quietFrames, padding, fade;
    double relative, floor, ceiling;
};

// A voice source shared by the voices of a batch that play the same sample from
// the same position at the same step, with the same loop and pitch ramp: their
// resampled source (render.cu:63-100) depends only on the frames elapsed since the
// voice began, so it is rendered once per batch and each voice reads it.
struct SharedSource {
    long long offset;                   // float offset of the source's frames in BatchView::shared
    int voice;                          // a voice playing it (its span fields define the source)
    int frames;                         // frames rendered; a voice's later frames are silent
};

// Per voice: where its shared source starts (-1: resampled inline) and how many
// of its frames the shared source covers.
struct SharedRef {
    long long offset;
    int frames, pad;
};

// Everything one synthesis pass reads, as device pointers.
struct BatchView {
    const float* bank;
    const float* sinc;                  // phase-major [2049][48]
    const cs_voice_span* voices;
    const cs_control_point* points;
    const cs_voice_modulation* modulation;
    const JobInfo* jobs;
    const MixTile* tiles;
    const int* indices;
    const int* blockJob;                // job of each 1024-frame block
    const int* windowJob;               // job of each tail window
    ChainState* states;
    float* filtered;
    double* phase;
    void* mix;                          // float2 (natural) or short2
    int* error;                         // set by kernels whose bounded waits ran out
    float* shared;                      // shared voice sources (mono: 1 float per frame, stereo: 2)
    const SharedRef* sharedRefs;        // per voice (null when no source is shared)
    int jobCount;
    int inlineVoices;                   // some voice has no filter chain (the mix renders it)
};

struct SegmentView {
    int first, end;                     // job-local frame range, 1024-aligned
    const uint64_t* scratchOffset;      // per voice: float offset into `filtered`
    const uint64_t* phaseOffset;        // per voice: offset into `phase`
    const int* chains;                  // heads of general chains active in this segment
    int chainCount;
    const int* simple;                  // heads of single-slot chains, longest first
    int simpleCount;
    const uint64_t* targetOffset;       // per voice: float offset of its filter targets
    const int2* sourceTiles;            // (span, first frame) of 256-frame source tiles
    int sourceTileCount;
    const int* pitchChains;
    int pitchCount;
    const int* blocks;                  // mix blocks in this segment
    int blockCount;
};

// Quality-gate / group-volume inputs of one job (the reference's AudioJob,
// src/cuda/render_types.h:116-118): frames of the melody body measured (0: none),
// its first body window and first onset in the batch arrays, and its onset count.
struct AssessJob {
    int bodyFrames, bodyFirst, onsetFirst, onsetCount;
};

// Body windows are 250 ms (5 quality windows) restarting every 2 s
// (src/cuda/quality.cu:13-19).
struct BodyGeometry {
    int chunk, span, perChunk;
    __host__ __device__ int windowOf(int frame) const { return frame / chunk * perChunk + frame % chunk / span; }
    __host__ __device__ int start(int window) const { return window / perChunk * chunk + window % perChunk * span; }
    __host__ __device__ int windows(int frames) const      // windows covering [0, frames)
    {
        return frames / chunk * perChunk + (frames % chunk + span - 1) / span;
    }
};

inline BodyGeometry bodyGeometry(const cs_audio_config& config)
{
    BodyGeometry g{2 * config.rate, 5 * config.window, 0};
    g.perChunk = (g.chunk + g.span - 1) / g.span;
    return g;
}

// Per-job reductions of the block-parallel tail searches: the first 1024-frame
// block that ends the natural search (2 * block + 1 when it is non-finite, else
// 2 * block; INT_MAX when none), the peak of the blocks before it (float bits),
// the loudest tail window's power (double bits) and the last loud window.
struct JobScan {
    int stop, peak, last, pad;
    unsigned long long maxPower;
};

struct FinishView {
    JobScan* scans;                     // one per job
    StereoStats* stereo;
    MonoStats* windows;
    short* mono;
    short* packed;
    cs_tail_result* results;
    int blockCount, windowCount;
    // Body power per window, accumulated by finalizeKernel from the samples it
    // writes (null when neither the quality gate nor group volume is on).
    unsigned long long* bodyPower;
    const AssessJob* assess;
    BodyGeometry body;
};

// The assessment stage (src/cuda/quality.cu): onset levels, verdicts, group gains.
struct AssessView {
    const AssessJob* jobs;
    const int* onsets;                  // onset frames, jobs concatenated
    const int* onsetJob;                // job of each onset
    const unsigned long long* bodyPower;
    unsigned long long* onsetPower;     // loudest 50 ms window after each onset
    cs_audio_config config;
    BodyGeometry body;
    int jobCount, onsetCount;
};

// Accepted-PCM packing (layoutAccepted + packAccepted, quality.cu:211-280): drops
// rejected jobs, applies group gains and re-measures gained jobs.
struct PackView {
    const int* blockJob;                // job of each 1024-frame block
    const int* jobBlockFirst;           // first block of each job
    cs_tail_result* results;
    uint64_t* sourceOffset;             // per job: its offset in `source` (set by the layout)
    const short* source;
    short* output;
    int jobCount, blockCount;
};

void buildSincTable(float* phaseMajor);   // host: 2049 x 48 floats

void launchScan(const BatchView& b, StereoStats* stats, int blocks, cudaStream_t stream);
// Source tiles (span, first frame) every kSourceTile frames of each run
// (span, first frame, end frame, first tile).
void launchExpandTiles(const int4* runs, int count, int2* tiles, cudaStream_t stream);
void launchPitch(const BatchView& b, const SegmentView& s, cudaStream_t stream);
// The mix tiles' voice lists: for each unit (job, chunk of kIndexChunkTiles tiles)
// the tiles' ranges into `indices` and, per tile, the job's overlapping spans in
// span order.
void launchTileIndex(const BatchView& b, const JobSpans* spans, const int2* units, int unitCount, MixTile* tiles,
                     int* indices, cudaStream_t stream);
// Renders the shared voice sources: `tiles` holds (source, first frame) every
// kSourceTile frames.
int launchSharedSources(const BatchView& b, const SharedSource* sources, const int2* tiles, int tileCount,
                        cudaStream_t stream);
int launchSources(const BatchView& b, const SegmentView& s, cudaStream_t stream);
int launchRecurrences(const BatchView& b, const SegmentView& s, cudaStream_t stream);
int launchGeneralChains(const BatchView& b, const SegmentView& s, cudaStream_t stream);
// `deferred`: device scratch of 1 + blocks ints for the blocks the lean mix pass
// leaves to the general one.
// Returns the kernels launched.
int launchMix(const BatchView& b, const SegmentView& s, bool natural, StereoStats* stats, int* deferred,
              cudaStream_t stream);
int launchFinish(const BatchView& b, const FinishView& f, bool natural, bool quality, const TailConfig& tail,
                 cudaStream_t stream);
// Onset levels (quality gate only) and per-job verdicts on the finished PCM.
int launchMeasure(const AssessView& a, cs_tail_result* results, const short* pcm, bool natural, cudaStream_t stream);
// Group gains for volume groups given as job ranges into `results`.
int launchMatch(const int2* groups, int count, int minimum, cs_tail_result* results, cudaStream_t stream);
int launchPack(const PackView& p, bool natural, cudaStream_t stream);

} // namespace cs
