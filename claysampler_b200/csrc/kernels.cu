// Synthesis and finishing kernels of the batch voice-render path (sm_100a).
//
//  chainKernel   one warp per voice chain (the spans of one note that share filter
//                state): 32 lanes resample, envelope and modulate 32 frames and
//                evaluate the per-frame filter targets in parallel; lanes 0/1 then
//                run the serial coefficient smoothing and biquad cascade for the left
//                and right channel.  Fuses the reference's renderFilterSources and
//                applyVoiceFilters (src/cuda/render.cu:195-220, 338-456).
//  mixKernel     one CTA per 1024-frame tail block: each thread sums the block's
//                overlapping voices for its frames in span order (renderTiles,
//                render.cu:458-523) and the CTA reduces the block's power and peak
//                in the same pass (scanStereo, src/cuda/tail.cu:54-81).
//  finishing     warp-per-job searches and block-parallel PCM passes restating
//                src/cuda/tail.cu:83-291.
#include "kernels.cuh"
#include "voice_math.cuh"

#include <climits>
#include <cmath>
#include <cstdio>
#include <initializer_list>
#include <mutex>

namespace cs {

// ---- sinc table (src/cuda/renderer.cpp:347-376) -----------------------------------

void buildSincTable(float* phaseMajor)
{
    constexpr double beta = 8.5, pi = 3.14159265358979323846;
    const auto besselI0 = [](double value) {
        double sum = 1, term = 1;
        for (int i = 1; i < 30; ++i) {
            term *= value * value / (4 * i * i);
            sum += term;
            if (term < 1e-14)
                break;
        }
        return sum;
    };
    const double norm = besselI0(beta);
    for (int phase = 0; phase <= kPhases; ++phase) {
        for (int tap = 0; tap < kTaps; ++tap) {
            const double x = tap - 23 - double(phase) / kPhases;
            const double f = x / 24;
            const double window = besselI0(beta * std::sqrt(1 - f * f)) / norm;
            phaseMajor[size_t(phase) * kTaps + tap] =
                static_cast<float>(window * (x == 0 ? 1 : std::sin(pi * x) / (pi * x)));
        }
    }
}

// ---- variable pitch (src/cuda/render.cu:222-274) ----------------------------------

__global__ void pitchKernel(BatchView b, SegmentView s)
{
    const int t = int(blockIdx.x * blockDim.x + threadIdx.x);
    if (t >= s.pitchCount)
        return;
    const int head = s.pitchChains[t];
    const cs_voice_span* voices = b.voices;
    if (!voices[head].variablePitch)
        return;
    ChainState& state = b.states[head];
    double position = state.pitchInitialized ? state.position : voices[head].position;
    int previousLoopEnd = state.previousLoopEnd, previousLoopStart = state.previousLoopStart;
    for (int span = head; span >= 0; span = voices[span].nextFilteredSpan) {
        const cs_voice_span& v = voices[span];
        if (v.end <= s.first || v.begin >= s.end)
            continue;
        const bool resumed = state.pitchInitialized && state.pitchSpan == span;
        if (!resumed && !v.loopEnd && previousLoopEnd > 0 && position >= previousLoopEnd)
            position = previousLoopStart + fmod(position - previousLoopStart,
                                                double(previousLoopEnd - previousLoopStart));
        previousLoopEnd = v.loopEnd;
        previousLoopStart = v.loopFirst;
        const double slope = exp(v.pitchSlope);
        double step = resumed ? state.step : v.step;
        const int start = max(v.begin, s.first), stop = min(v.end, s.end);
        double* out = b.phase + s.phaseOffset[span];
        for (int frame = start; frame < stop; ++frame) {
            out[frame - start] = position;
            float cents = 0;
            float depth = v.extraEnvelope[1].depth;
            for (int j = v.firstModulation; j < v.firstModulation + v.modulationCount; ++j) {
                const cs_voice_modulation m = b.modulation[j];
                if (m.target == CS_MOD_PITCH)
                    cents += bindingAt(m, b.points, frame);
                if (m.target == CS_MOD_PITCHEG_DEPTH)
                    depth += bindingAt(m, b.points, frame);
            }
            if (v.activeEnvelope[1])
                cents += depth * envelopeAt(v.extraEnvelope[1], frame);
            position += step * exp2f(fminf(24000.f, fmaxf(-24000.f, cents)) / 1200);
            step *= slope;
        }
        state.pitchInitialized = 1;
        state.pitchSpan = span;
        state.position = position;
        state.step = step;
        state.previousLoopEnd = previousLoopEnd;
        state.previousLoopStart = previousLoopStart;
    }
}

// ---- fused source + filter chains ---------------------------------------------------

constexpr int kChainWarps = 8;
constexpr int kChunk = 32;

struct ChainShared {
    float2 source[kChunk];
    float2 output[kChunk];
    Biquad target[kChunk][CS_FILTER_SLOTS];
};

__global__ void __launch_bounds__(kChainWarps * 32) chainKernel(BatchView b, SegmentView s)
{
    __shared__ ChainShared shared[kChainWarps];
    const int warp = int(threadIdx.x >> 5), lane = int(threadIdx.x & 31);
    const int chain = int(blockIdx.x) * kChainWarps + warp;
    if (chain >= s.chainCount)
        return;
    ChainShared& sh = shared[warp];
    const int head = s.chains[chain];
    const cs_voice_span* voices = b.voices;
    bool filtered = false;
    for (int f = 0; f < CS_FILTER_SLOTS; ++f)
        filtered |= voices[head].filters[f].type != CS_FILTER_NONE;
    ChainState& state = b.states[head];

    // Serial state: lane c (c = 0, 1) owns channel c of every section.
    const int channel = lane;
    bool initialized = state.filterInitialized != 0;
    Biquad current[CS_FILTER_SLOTS];
    float z1[CS_FILTER_SLOTS][3], z2[CS_FILTER_SLOTS][3];
    if (filtered && lane < 2) {
        #pragma unroll
        for (int f = 0; f < CS_FILTER_SLOTS; ++f) {
            current[f] = {state.coefficients[f][0], state.coefficients[f][1], state.coefficients[f][2],
                          state.coefficients[f][3], state.coefficients[f][4]};
            #pragma unroll
            for (int k = 0; k < 3; ++k) {
                z1[f][k] = state.z1[f][k][channel];
                z2[f][k] = state.z2[f][k][channel];
            }
        }
    }

    for (int span = head; span >= 0; span = voices[span].nextFilteredSpan) {
        const cs_voice_span& v = voices[span];
        if (v.end <= s.first || v.begin >= s.end)
            continue;
        const int channels = v.channels;
        const int start = max(v.begin, s.first), stop = min(v.end, s.end);
        float* out = b.filtered + s.scratchOffset[span];
        const double* phase = v.variablePitch ? b.phase + s.phaseOffset[span] : nullptr;
        const int* tracks = v.filterControls;
        int sections[CS_FILTER_SLOTS];
        #pragma unroll
        for (int f = 0; f < CS_FILTER_SLOTS; ++f)
            sections[f] = filtered ? filterSections(v.filters[f].type) : 0;
        const bool moving = filtered && filterMoves(v, b.modulation);
        const float amount = 1 - expf(-1000.f / float(v.sampleRate));

        for (int base = start; base < stop; base += kChunk) {
            const int frame = base + lane;
            const int count = min(kChunk, stop - base);
            const bool needTargets = filtered && (moving || !initialized);
            if (lane < count) {
                const double position = phase ? phase[frame - start] : -1.0;
                const float pan = trackAt(b.points, tracks[2], tracks[3], frame);
                const float2 sample = voiceFrame(b.bank, b.sinc, v, b.points, b.modulation, pan, frame, true,
                                                 position);
                const float gain = jobGainAt(b.points, tracks, frame);
                sh.source[lane] = make_float2(sample.x * gain, sample.y * gain);
                if (needTargets)
                    filterTargets(v, b.points, b.modulation, frame, sh.target[lane]);
            }
            __syncwarp();
            if (filtered) {
                if (lane < channels) {
                    for (int i = 0; i < count; ++i) {
                        if (moving || !initialized) {
                            #pragma unroll
                            for (int f = 0; f < CS_FILTER_SLOTS; ++f) {
                                if (!sections[f])
                                    continue;
                                if (initialized) smoothToward(current[f], sh.target[i][f], amount);
                                else current[f] = sh.target[i][f];
                            }
                            initialized = true;
                        }
                        float x = channel == 0 ? sh.source[i].x : sh.source[i].y;
                        #pragma unroll
                        for (int f = 0; f < CS_FILTER_SLOTS; ++f) {
                            #pragma unroll
                            for (int k = 0; k < 3; ++k)
                                if (k < sections[f])
                                    x = biquadStep(x, current[f], z1[f][k], z2[f][k]);
                        }
                        if (channel == 0) sh.output[i].x = x;
                        else sh.output[i].y = x;
                    }
                }
                // Lanes without a channel track the flag the serial lanes advanced.
                initialized = initialized || moving || count > 0;
                __syncwarp();
            } else if (lane < count) {
                sh.output[lane] = sh.source[lane];
            }
            __syncwarp();
            if (lane < count) {
                const float2 y = sh.output[lane];
                float* dst = out + size_t(frame - start) * channels;
                dst[0] = y.x;
                if (channels == 2)
                    dst[1] = y.y;
            }
            __syncwarp();
        }
    }
    if (filtered && lane < 2) {
        if (lane == 0)
            state.filterInitialized = initialized;
        #pragma unroll
        for (int f = 0; f < CS_FILTER_SLOTS; ++f) {
            if (lane == 0) {
                state.coefficients[f][0] = current[f].b0;
                state.coefficients[f][1] = current[f].b1;
                state.coefficients[f][2] = current[f].b2;
                state.coefficients[f][3] = current[f].a1;
                state.coefficients[f][4] = current[f].a2;
            }
            #pragma unroll
            for (int k = 0; k < 3; ++k) {
                state.z1[f][k][channel] = z1[f][k];
                state.z2[f][k][channel] = z2[f][k];
            }
        }
    }
}

// ---- single-slot chains: parallel sources, one recurrence per lane -------------------
//
// Chains whose spans all filter through one main slot with one filter type run in
// two kernels.  sourceKernel renders every voice frame in parallel (256-frame
// tiles, each thread a frame at a time) and, for moving filters, the per-frame target
// coefficients in a 3-float form: for the low/high/band-pass, notch and one-pole
// designs the remaining coefficients are exact multiples (x2, -1, equal) of these
// three, and the component-wise smoothing preserves those relations bit for bit.
// recurrenceKernel then runs each chain's smoothing and biquad cascade serially,
// two lanes per chain (one per channel), from chunks staged in shared memory.

__device__ __forceinline__ int activeSlot(const cs_voice_span& v)
{
    for (int f = 0; f < 2; ++f)
        if (v.filters[f].type != CS_FILTER_NONE)
            return f;
    return -1;
}

struct Compact {
    float c0, c1, c2;
};

__device__ __forceinline__ Compact compactOf(int type, const Biquad& q)
{
    (void)type;
    return {q.b0, q.a1, q.a2};
}

__device__ __forceinline__ Biquad expand(int type, const Compact& c)
{
    switch (type) {
    case CS_FILTER_LOW1: return {c.c0, 0.f, 0.f, c.c1, 0.f};
    case CS_FILTER_HIGH1: return {c.c0, -c.c0, 0.f, c.c1, 0.f};
    case CS_FILTER_HIGH2: case CS_FILTER_HIGH4: case CS_FILTER_HIGH6:
        return {c.c0, -2 * c.c0, c.c0, c.c1, c.c2};
    case CS_FILTER_BAND2: case CS_FILTER_BAND4: case CS_FILTER_BAND6:
        return {c.c0, 0.f, -c.c0, c.c1, c.c2};
    case CS_FILTER_NOTCH2: return {c.c0, c.c1, c.c0, c.c1, c.c2};
    default: return {c.c0, 2 * c.c0, c.c0, c.c1, c.c2};
    }
}

// One voice-frame of a source tile.
__device__ __forceinline__ void sourceFrame(const BatchView& b, const SegmentView& s, int span, int frame)
{
    const cs_voice_span& v = b.voices[span];
    const int start = max(v.begin, s.first);
    const int* tracks = v.filterControls;
    const float pan = trackAt(b.points, tracks[2], tracks[3], frame);
    const uint64_t targets = s.targetOffset[span];
    const int f = targets == kNoTargets ? -1 : activeSlot(v);
    // voiceFrame and filterTargetSlot with one walk over the bindings; the filter
    // targets first, so that their sums are dead before the voice is rendered.
    const float level = envelopeAt(v, frame);
    const SourceMods mods = sourceMods(v, b.points, b.modulation, level, pan, frame, f);
    if (f >= 0 && (mods.moving || frame == v.begin)) {
        const Compact c = compactOf(v.filters[f].type, filterFromMods(v, f, mods.filter, frame));
        if (mods.moving) {
            const int rel = frame - start;
            float* out = b.filtered + targets + size_t(rel / kRecChunkFrames) * 3 * kRecChunkFrames + rel % kRecChunkFrames;
            out[0] = c.c0;
            out[kRecChunkFrames] = c.c1;
            out[2 * kRecChunkFrames] = c.c2;
        } else {
            float* out = b.filtered + targets;
            out[0] = c.c0;
            out[1] = c.c1;
            out[2] = c.c2;
        }
    }
    const double position = v.variablePitch ? b.phase[s.phaseOffset[span] + (frame - start)] : -1.0;
    const float2 sample = level <= 0 ? make_float2(0.f, 0.f)
                                     : voiceOutput(b.bank, b.sinc, v, mods.voice, frame, true, position);
    const float gain = jobGainAt(b.points, tracks, frame);
    float* dst = b.filtered + s.scratchOffset[span] + size_t(frame - start) * v.channels;
    dst[0] = sample.x * gain;
    if (v.channels == 2)
        dst[1] = sample.y * gain;
}

// Shared-memory carveout (percent of the maximum) of the source and recurrence
// kernels, which run side by side: one setting lets a recurrence CTA (164 KB of
// staged chunks) start on an SM that holds source CTAs, where different settings
// make the SM drain first.  75 % leaves the source kernel 60 KB and more of L1;
// measured on the 64-job step against 100 % and the default.
constexpr int kOverlapCarveout = 75;

// A CTA of kSourceThreads renders one 256-frame source tile, each thread every
// kSourceThreads-th frame.  Small CTAs matter when recurrences run beside the
// sources: an SM holds at most 64 warps, and each 2-warp recurrence CTA then
// displaces one source CTA.
__global__ void __launch_bounds__(kSourceThreads, 2048 / kSourceThreads) sourceKernel(BatchView b, SegmentView s)
{
    const int2 tile = s.sourceTiles[blockIdx.x];
    const int end = min(min(b.voices[tile.x].end, s.end), tile.y + kSourceTile);
    #pragma unroll 1
    for (int frame = tile.y + int(threadIdx.x); frame < end; frame += kSourceThreads)
        sourceFrame(b, s, tile.x, frame);
}

// ---- TMA-staged serial recurrences --------------------------------------------------
//
// Two lanes per chain (one per channel), 16 chains per warp.  Each chain keeps
// kRecBuffers chunks of kRecChunk frames in shared memory, filled by
// cp.async.bulk copies that its leader lane issues and that complete on the chain's
// own mbarriers, so the next chunk's sources and targets arrive while the current
// one runs through the smoothing and biquad recurrence.  The kernel's time is the
// longest chain's, which is bound by the instructions its warp issues per frame;
// large chunks keep the per-chunk work (wait, cursor advance, copy issue) small
// beside the per-frame work.  Waits are bounded: a wait that runs out sets the
// batch's error flag and the lane stops.

#ifndef CS_REC_CHUNK
#define CS_REC_CHUNK 128
#endif
constexpr int kRecChunk = CS_REC_CHUNK;                               // staged frames, a multiple of 32
static_assert(kRecChunk % kRecChunkFrames == 0, "staged chunks hold whole target plane groups");
constexpr int kRecBuffers = 2;
constexpr int kRecBuffer = kRecChunk * 2 * 4 + kRecChunk * 3 * 4;     // sources, then target plane groups
constexpr int kRecChainBytes = kRecBuffers * kRecBuffer + 16;         // skew: conflict-free LDS.128
constexpr int kRecChains = 16;                                        // per warp: lane = 2 * chain + channel
constexpr int kRecWarps = 2;
constexpr int kRecThreads = 32 * kRecWarps;
static_assert(kRecWarps * kRecChains == kRecChainsPerCta, "chains per recurrence CTA");
constexpr long long kWaitLimit = 1ll << 24;

__device__ __forceinline__ uint32_t sharedAddress(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void barrierInit(uint64_t* bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sharedAddress(bar)) : "memory");
}

__device__ __forceinline__ void barrierExpect(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sharedAddress(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulkLoad(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(sharedAddress(dst)), "l"(src), "r"(bytes), "r"(sharedAddress(bar)) : "memory");
}

__device__ __forceinline__ bool barrierTryWait(uint64_t* bar, uint32_t parity)
{
    uint32_t done;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                 " selp.u32 %0, 1, 0, p;\n}" : "=r"(done) : "r"(sharedAddress(bar)), "r"(parity) : "memory");
    return done != 0;
}

__device__ __forceinline__ bool barrierWait(uint64_t* bar, uint32_t parity)
{
    for (long long i = 0; i < kWaitLimit; ++i)
        if (barrierTryWait(bar, parity))
            return true;
    return false;
}

__device__ __forceinline__ uint32_t round16(uint32_t bytes) { return (bytes + 15u) & ~15u; }

// One channel of one chain through staged frames [first, count) of a 32-frame
// chunk.  Sources are interleaved per frame (stereo) and targets are planar, so
// aligned groups of four frames need one or two 128-bit loads each; Type fixes
// how the two derived numerator taps follow from the three carried coefficients.
template <int Type, int Sections, bool Moving, bool Stereo>
__device__ __forceinline__ void recurChunk(const float* __restrict__ frames, const float* __restrict__ targets,
                                           float* __restrict__ out, int first, int count, int channel,
                                           float amount, Compact& c, float* z1, float* z2)
{
    constexpr int stride = Stereo ? 2 : 1;
    const auto frameStep = [&](float x, float t0, float t1, float t2) {
        if (Moving) {
            c.c0 = fmaf(amount, t0 - c.c0, c.c0);
            c.c1 = fmaf(amount, t1 - c.c1, c.c1);
            c.c2 = fmaf(amount, t2 - c.c2, c.c2);
        }
        const Biquad q = expand(Type, c);
        #pragma unroll
        for (int sct = 0; sct < Sections; ++sct)
            x = biquadStep(x, q, z1[sct], z2[sct]);
        return x;
    };
    int i = first;
    for (; i < count && (i & 3); ++i) {
        const float x = frames[stride * i + channel];
        out[stride * i] = frameStep(x, Moving ? targets[i] : 0.f, Moving ? targets[kRecChunkFrames + i] : 0.f,
                                    Moving ? targets[2 * kRecChunkFrames + i] : 0.f);
    }
    // Groups of kGroup frames: the coefficient smoothing of the whole group runs
    // first (it does not depend on the audio), then the biquad steps, so the
    // warp's in-order issue always has independent work between dependent steps.
    constexpr int kGroup = 8;
    for (; i + kGroup <= count; i += kGroup) {
        float x[kGroup];
        #pragma unroll
        for (int k = 0; k < kGroup; ++k)
            x[k] = frames[stride * (i + k) + channel];
        Biquad q[kGroup];
        #pragma unroll
        for (int k = 0; k < kGroup; k += 4) {
            float4 t0 = make_float4(0, 0, 0, 0), t1 = t0, t2 = t0;
            if (Moving) {
                t0 = *reinterpret_cast<const float4*>(targets + i + k);
                t1 = *reinterpret_cast<const float4*>(targets + kRecChunkFrames + i + k);
                t2 = *reinterpret_cast<const float4*>(targets + 2 * kRecChunkFrames + i + k);
            }
            const float a0[4] = {t0.x, t0.y, t0.z, t0.w}, a1[4] = {t1.x, t1.y, t1.z, t1.w};
            const float a2[4] = {t2.x, t2.y, t2.z, t2.w};
            #pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (Moving) {
                    c.c0 = fmaf(amount, a0[j] - c.c0, c.c0);
                    c.c1 = fmaf(amount, a1[j] - c.c1, c.c1);
                    c.c2 = fmaf(amount, a2[j] - c.c2, c.c2);
                }
                q[k + j] = expand(Type, c);
            }
        }
        #pragma unroll
        for (int k = 0; k < kGroup; ++k) {
            float y = x[k];
            #pragma unroll
            for (int sct = 0; sct < Sections; ++sct)
                y = biquadStep(y, q[k], z1[sct], z2[sct]);
            out[stride * (i + k)] = y;
        }
    }
    for (; i < count; ++i) {
        const float x = frames[stride * i + channel];
        out[stride * i] = frameStep(x, Moving ? targets[i] : 0.f, Moving ? targets[kRecChunkFrames + i] : 0.f,
                                    Moving ? targets[2 * kRecChunkFrames + i] : 0.f);
    }
}

template <int Type, bool Stereo>
__device__ __forceinline__ void recurSections(const float* frames, const float* targets, float* out, int first,
                                              int count, int channel, int sections, bool moving, float amount,
                                              Compact& c, float* z1, float* z2)
{
    if (moving) {
        if (sections == 1) recurChunk<Type, 1, true, Stereo>(frames, targets, out, first, count, channel, amount, c, z1, z2);
        else if (sections == 2) recurChunk<Type, 2, true, Stereo>(frames, targets, out, first, count, channel, amount, c, z1, z2);
        else recurChunk<Type, 3, true, Stereo>(frames, targets, out, first, count, channel, amount, c, z1, z2);
    } else {
        if (sections == 1) recurChunk<Type, 1, false, Stereo>(frames, targets, out, first, count, channel, amount, c, z1, z2);
        else if (sections == 2) recurChunk<Type, 2, false, Stereo>(frames, targets, out, first, count, channel, amount, c, z1, z2);
        else recurChunk<Type, 3, false, Stereo>(frames, targets, out, first, count, channel, amount, c, z1, z2);
    }
}

template <bool Stereo>
__device__ __forceinline__ void recurDispatch(int type, const float* frames, const float* targets, float* out,
                                              int first, int count, int channel, int sections, bool moving,
                                              float amount, Compact& c, float* z1, float* z2)
{
    switch (type) {
    case CS_FILTER_LOW1:
        recurSections<CS_FILTER_LOW1, Stereo>(frames, targets, out, first, count, channel, sections, moving, amount, c, z1, z2);
        break;
    case CS_FILTER_HIGH1:
        recurSections<CS_FILTER_HIGH1, Stereo>(frames, targets, out, first, count, channel, sections, moving, amount, c, z1, z2);
        break;
    case CS_FILTER_HIGH2: case CS_FILTER_HIGH4: case CS_FILTER_HIGH6:
        recurSections<CS_FILTER_HIGH2, Stereo>(frames, targets, out, first, count, channel, sections, moving, amount, c, z1, z2);
        break;
    case CS_FILTER_BAND2: case CS_FILTER_BAND4: case CS_FILTER_BAND6:
        recurSections<CS_FILTER_BAND2, Stereo>(frames, targets, out, first, count, channel, sections, moving, amount, c, z1, z2);
        break;
    case CS_FILTER_NOTCH2:
        recurSections<CS_FILTER_NOTCH2, Stereo>(frames, targets, out, first, count, channel, sections, moving, amount, c, z1, z2);
        break;
    default:
        recurSections<CS_FILTER_LOW2, Stereo>(frames, targets, out, first, count, channel, sections, moving, amount, c, z1, z2);
        break;
    }
}

// Per-span constants of a chain cursor, loaded once when the cursor enters a span.
struct SpanRun {
    int span, pos, stop, start, channels, sections;
    int moving;
    float amount;
    const float* src;                   // span's source frames in the segment scratch
    const float* tgt;                   // span's filter targets (moving: per frame)
};

__device__ __forceinline__ SpanRun enterRun(const BatchView& b, const SegmentView& s, int from, int fslot)
{
    const cs_voice_span* voices = b.voices;
    for (int at = from; at >= 0; at = voices[at].nextFilteredSpan) {
        const cs_voice_span& v = voices[at];
        if (v.begin >= s.end)
            break;
        if (v.end <= s.first)
            continue;
        SpanRun r;
        r.span = at;
        r.start = max(v.begin, s.first);
        r.pos = r.start;
        r.stop = min(v.end, s.end);
        r.channels = v.channels;
        r.sections = filterSections(v.filters[fslot].type);
        const uint64_t toff = s.targetOffset[at];
        r.moving = toff != kNoTargets && filterMoves(v, b.modulation);
        r.amount = 1 - expf(-1000.f / float(v.sampleRate));
        r.src = b.filtered + s.scratchOffset[at];
        r.tgt = b.filtered + (toff == kNoTargets ? 0 : toff);
        return r;
    }
    SpanRun none{};
    none.span = -1;
    return none;
}

__device__ __forceinline__ void advanceRun(const BatchView& b, const SegmentView& s, SpanRun& r, int fslot)
{
    r.pos += min(kRecChunk, r.stop - r.pos);
    if (r.pos >= r.stop)
        r = enterRun(b, s, b.voices[r.span].nextFilteredSpan, fslot);
}

__global__ void __launch_bounds__(kRecThreads, 1) recurrenceKernel(BatchView b, SegmentView s, int* error)
{
    extern __shared__ __align__(16) unsigned char staged[];
    __shared__ __align__(8) uint64_t bars[kRecWarps * kRecChains][kRecBuffers];
    const int lane = int(threadIdx.x & 31), warp = int(threadIdx.x >> 5);
    const int local = warp * kRecChains + (lane >> 1);
    const int channel = lane & 1;
    const int chain = int(blockIdx.x) * kRecWarps * kRecChains + local;
    const cs_voice_span* voices = b.voices;
    int head = -1, fslot = -1, type = CS_FILTER_NONE;
    if (chain < s.simpleCount) {
        head = s.simple[chain];
        fslot = activeSlot(voices[head]);
        if (fslot >= 0)
            type = voices[head].filters[fslot].type;
    }
    // Pitch-only chains and mono chains' right lanes have nothing to run.
    const bool leader = channel == 0 && fslot >= 0;
    const bool active = fslot >= 0 && (channel == 0 || voices[head].channels == 2);
    unsigned char* region = staged + size_t(local) * kRecChainBytes;
    if (leader)
        for (int k = 0; k < kRecBuffers; ++k)
            barrierInit(&bars[local][k]);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncwarp();
    if (!active)
        return;
    // Both lanes of a stereo chain read each staged buffer before it is refilled.
    const unsigned pair = (voices[head].channels == 2 ? 3u : 1u) << (lane & ~1);
    ChainState& state = b.states[head];
    bool initialized = state.filterInitialized != 0;
    Compact c{state.coefficients[fslot][0], state.coefficients[fslot][3], state.coefficients[fslot][4]};
    float z1[3], z2[3];
    #pragma unroll
    for (int k = 0; k < 3; ++k) {
        z1[k] = state.z1[fslot][k][channel];
        z2[k] = state.z2[fslot][k][channel];
    }

    SpanRun consume = enterRun(b, s, head, fslot);
    SpanRun next = consume;
    const auto issue = [&](int slot) {
        const int count = min(kRecChunk, next.stop - next.pos);
        const int rel = next.pos - next.start;
        const uint32_t srcBytes = round16(uint32_t(count * next.channels) * 4u);
        // Only the plane groups the chunk's frames use (the span's last may be partial).
        const uint32_t tgtBytes = next.moving ? uint32_t((count + kRecChunkFrames - 1) / kRecChunkFrames) *
            uint32_t(3 * kRecChunkFrames * 4) : 0u;
        unsigned char* buffer = region + slot * kRecBuffer;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        barrierExpect(&bars[local][slot], srcBytes + tgtBytes);
        bulkLoad(buffer, next.src + size_t(rel) * next.channels, srcBytes, &bars[local][slot]);
        if (tgtBytes)
            bulkLoad(buffer + kRecChunk * 2 * 4, next.tgt + size_t(rel / kRecChunkFrames) * 3 * kRecChunkFrames,
                     tgtBytes, &bars[local][slot]);
    };
    uint32_t phases = 0;                 // bit k: parity of buffer k's next completion
    uint32_t inflight = 0;               // bit k: buffer k has a copy issued and not yet waited for
    for (int slot = 0; slot < kRecBuffers && next.span >= 0; ++slot) {
        if (leader)
            issue(slot);
        inflight |= 1u << slot;
        advanceRun(b, s, next, fslot);
    }
    int slot = 0;
    while (consume.span >= 0) {
        if (!barrierWait(&bars[local][slot], (phases >> slot) & 1u)) {
            // Give up: flag the batch, issue nothing more, and wait (bounded) for
            // the copies still in flight into this chain's buffers before leaving.
            atomicExch(error, 1);
            for (int k = 0; k < kRecBuffers; ++k)
                if (inflight >> k & 1u)
                    barrierWait(&bars[local][k], (phases >> k) & 1u);
            return;
        }
        phases ^= 1u << slot;
        inflight &= ~(1u << slot);
        const int count = min(kRecChunk, consume.stop - consume.pos);
        const int rel = consume.pos - consume.start;
        const int sections = consume.sections;
        const bool moving = consume.moving != 0;
        const int stride = consume.channels;
        const float* frames = reinterpret_cast<const float*>(region + slot * kRecBuffer);
        const float* targets = frames + kRecChunk * 2;
        float* out = const_cast<float*>(consume.src) + size_t(rel) * stride + channel;
        if (sections) {
            int first = 0;
            if (!initialized) {
                // The chain's first frame takes its targets without smoothing.
                if (moving)
                    c = {targets[0], targets[kRecChunkFrames], targets[2 * kRecChunkFrames]};
                else
                    c = {consume.tgt[0], consume.tgt[1], consume.tgt[2]};
                initialized = true;
                const Biquad q = expand(type, c);
                float x = frames[channel];
                #pragma unroll
                for (int k = 0; k < 3; ++k)
                    if (k < sections)
                        x = biquadStep(x, q, z1[k], z2[k]);
                out[0] = x;
                first = 1;
            }
            // One target plane group per 32 frames.
            for (int half = 0; half * kRecChunkFrames < count; ++half) {
                const int base = half * kRecChunkFrames;
                const int n = min(kRecChunkFrames, count - base);
                const float* planes = targets + half * 3 * kRecChunkFrames;
                if (stride == 2)
                    recurDispatch<true>(type, frames + 2 * base, planes, out + 2 * base, half ? 0 : first, n, channel,
                                        sections, moving, consume.amount, c, z1, z2);
                else
                    recurDispatch<false>(type, frames + base, planes, out + base, half ? 0 : first, n, channel,
                                         sections, moving, consume.amount, c, z1, z2);
            }
        } else {
            initialized = true;
        }
        advanceRun(b, s, consume, fslot);
        __syncwarp(pair);
        if (next.span >= 0) {
            if (leader)
                issue(slot);
            inflight |= 1u << slot;
            advanceRun(b, s, next, fslot);
        }
        slot = slot + 1 == kRecBuffers ? 0 : slot + 1;
    }
    if (channel == 0) {
        state.filterInitialized = initialized;
        const Biquad q = expand(type, c);
        float* coeff = state.coefficients[fslot];
        coeff[0] = q.b0; coeff[1] = q.b1; coeff[2] = q.b2; coeff[3] = q.a1; coeff[4] = q.a2;
    }
    #pragma unroll
    for (int k = 0; k < 3; ++k) {
        state.z1[fslot][k][channel] = z1[k];
        state.z2[fslot][k][channel] = z2[k];
    }
}

// ---- shared voice sources ------------------------------------------------------------
//
// The voice source of render.cu:63-100 (position, loop wrap and crossfade, 48-tap
// sinc) of every frame of every shared source, stored as one float (mono) or two
// (stereo); the mix then reads it for every voice that plays the source.  A
// persistent CTA per SM first copies the half sinc table (phases 0-1024, 213 KB)
// into shared memory, where each lane's scattered row reads cost a shared-memory
// access instead of an L2 round trip, then takes 256-frame tiles, a thread per
// frame, consecutive threads on consecutive frames.
constexpr int kSharedSourceThreads = 1024;
constexpr size_t kSharedSincBytes = size_t(kSharedSincRows) * kSharedSincStride * sizeof(float);

__global__ void __launch_bounds__(kSharedSourceThreads, 1) sharedSourceKernel(BatchView b,
                                                                               const SharedSource* __restrict__ sources,
                                                                               const int2* __restrict__ tiles,
                                                                               int tileCount)
{
    extern __shared__ __align__(16) float table[];
    for (int i = int(threadIdx.x); i < kSharedSincRows * (kTaps / 4); i += kSharedSourceThreads) {
        const int row = i / (kTaps / 4), quad = i % (kTaps / 4);
        reinterpret_cast<float4*>(table + row * kSharedSincStride)[quad] =
            __ldg(reinterpret_cast<const float4*>(b.sinc + size_t(row) * kTaps) + quad);
    }
    __syncthreads();
    const SharedSincRows rows{table};
    const long long items = (long long)tileCount * kSourceTile;
    for (long long item = (long long)blockIdx.x * kSharedSourceThreads + threadIdx.x; item < items;
         item += (long long)gridDim.x * kSharedSourceThreads) {
        const int2 tile = tiles[item / kSourceTile];
        const SharedSource source = sources[tile.x];
        const int i = tile.y + int(item % kSourceTile);
        if (i >= source.frames)
            continue;
        const cs_voice_span& v = b.voices[source.voice];
        const float2 x = voiceSourceRows<true>(b.bank, rows, v, v.begin + i, -1.0);
        float* out = b.shared + source.offset;
        if (v.channels == 2)
            reinterpret_cast<float2*>(out)[i] = x;
        else
            out[i] = x.x;
    }
}

// ---- mix + block scan ----------------------------------------------------------------

constexpr int kMixThreads = 256;


// The block's power (sum) and peak (maximum) at once, one barrier; valid in
// thread 0.  `sums` and `peaks` hold a slot per warp and serve no other use.
__device__ __forceinline__ void blockStats(double& power, float& peak, double* sums, float* peaks)
{
    #pragma unroll
    for (int d = 16; d; d >>= 1) {
        power += __shfl_down_sync(0xffffffffu, power, d);
        const float other = __shfl_down_sync(0xffffffffu, peak, d);
        peak = other > peak ? other : peak;
    }
    const int warp = int(threadIdx.x >> 5), lane = int(threadIdx.x & 31);
    if (!lane) {
        sums[warp] = power;
        peaks[warp] = peak;
    }
    __syncthreads();
    if (warp == 0) {
        const bool held = lane < int(blockDim.x >> 5);
        power = held ? sums[lane] : 0.0;
        peak = held ? peaks[lane] : 0.f;
        #pragma unroll
        for (int d = 16; d; d >>= 1) {
            power += __shfl_down_sync(0xffffffffu, power, d);
            const float other = __shfl_down_sync(0xffffffffu, peak, d);
            peak = other > peak ? other : peak;
        }
    }
}

struct SumOp { template <class T> __device__ T operator()(T a, T b) const { return a + b; } };
struct MaxOp { template <class T> __device__ T operator()(T a, T b) const { return a > b ? a : b; } };
struct MinOp { __device__ int operator()(int a, int b) const { return a < b ? a : b; } };

// A tile's voice as the mix reads it: frame range, where its filtered frames
// start (in floats, relative to frame 0 of the job), its index and kind.
struct MixVoice {
    long long offset;                   // filtered (shared) + offset + frame * channels is the frame's first sample
    int begin, end, index, kind;        // kind: 0 unfiltered, 1 filtered stereo, 2 filtered mono,
                                        // 3 shared mono source, 4 shared stereo source, 5 / 6 as 3 / 4
                                        // with no modulation, no stereo matrix and the tile's pan fixed
    int sharedEnd;                      // kinds 3-6: frames from here on have a silent source
    float gainLeft, gainRight;          // kinds 5, 6: the voice's pan gains over the tile
    // Kinds 5, 6: the amplitude envelope's piece over the tile (EnvelopePiece),
    // the frame it counts from, its rate and its value.
    int piece, pieceFrame;
    float pieceRate, pieceValue;
};

// The pieces of an amplitude envelope (envelopeAt, render.cu:6-19), in the order
// its tests pick them.  Each piece holds over one interval of frames: a frame's
// piece follows from comparisons that each flip once as the frame grows, so a
// tile whose first and last frames share a piece has it for every frame.
enum EnvelopePiece : int {
    kPieceStart, kPieceAttack, kPieceHold, kPieceSustain, kPieceDecay, kPieceRelease, kPieceFade, kPieceAny
};

template <class Shape>
__device__ __forceinline__ int envelopePiece(const Shape& e, int frame)
{
    if (e.releaseStart >= 0 && frame >= e.releaseStart)
        return frame >= e.fadeStart ? kPieceFade : kPieceRelease;
    if (frame < e.attackStart) return kPieceStart;
    if (frame < e.holdStart) return kPieceAttack;
    if (frame < e.decayStart) return kPieceHold;
    return e.decayRate == 0 ? kPieceSustain : kPieceDecay;
}

// Stages the envelope of `m` over frames [first, last] as one piece when it has one.
template <class Shape>
__device__ __forceinline__ void stageEnvelope(MixVoice& m, const Shape& e, int first, int last)
{
    const int piece = envelopePiece(e, first);
    m.piece = piece == envelopePiece(e, last) ? piece : kPieceAny;
    m.pieceFrame = 0;
    m.pieceRate = m.pieceValue = 0.f;
    switch (m.piece) {
    case kPieceStart: m.pieceValue = e.start; break;
    case kPieceAttack: m.pieceFrame = e.attackStart; m.pieceRate = e.attackStep; m.pieceValue = e.start; break;
    case kPieceHold: m.pieceValue = 1.f; break;
    case kPieceSustain: m.pieceValue = e.sustain; break;
    case kPieceDecay: m.pieceFrame = e.decayStart; m.pieceRate = e.decayRate; m.pieceValue = e.sustain; break;
    case kPieceRelease:
        m.pieceFrame = e.releaseStart; m.pieceRate = e.releaseRate; m.pieceValue = e.releaseValue; break;
    case kPieceFade: m.pieceFrame = e.fadeStart; m.pieceRate = e.fadeStep; m.pieceValue = e.fadeValue; break;
    default: break;
    }
}

// envelopeAt through the staged piece: the same expression on the same fields.
__device__ __forceinline__ float envelopeOf(const MixVoice& m, const cs_voice_span* __restrict__ voices, int frame)
{
    switch (m.piece) {
    case kPieceStart:
    case kPieceHold:
    case kPieceSustain: return m.pieceValue;
    case kPieceAttack: return fminf(1.f, m.pieceValue + float(frame - m.pieceFrame + 1) * m.pieceRate);
    case kPieceDecay: return fmaxf(m.pieceValue, expf(float(frame - m.pieceFrame + 1) * m.pieceRate));
    case kPieceRelease: return m.pieceValue * expf(float(frame - m.pieceFrame + 1) * m.pieceRate);
    case kPieceFade: return fmaxf(0.f, m.pieceValue - float(frame - m.pieceFrame + 1) * m.pieceRate);
    default: return envelopeAt(voices[m.index], frame);
    }
}

// A job control track (CC7, CC11 or the channel pan) over one 256-frame tile.
// pointAt never decreases with the frame, so when the tile's first and last
// frames find the same point every frame between them does too, and the track's
// value there is that point's line: the expression trackAt evaluates, with the
// point's fields read once per tile.  Otherwise each frame looks its point up.
struct TileTrack {
    float value, step;
    int frame;                          // the point's frame; INT_MIN: look each frame up
    int low, high;                      // the track's points
};

__device__ __forceinline__ TileTrack tileTrackOf(const cs_control_point* __restrict__ points, int low, int high,
                                                 int first, int last)
{
    TileTrack t{0.f, 0.f, INT_MIN, low, high};
    const int at = pointAt(points, low, high, first);
    if (at == pointAt(points, low, high, last)) {
        t.value = __ldg(&points[at].value);
        t.step = __ldg(&points[at].step);
        t.frame = __ldg(&points[at].frame);
    }
    return t;
}

__device__ __forceinline__ float tileTrackAt(const TileTrack& t, const cs_control_point* __restrict__ points, int frame)
{
    if (t.frame == INT_MIN)
        return trackAt(points, t.low, t.high, frame);
    return fmaf(t.step, float(frame - t.frame), t.value);
}

// Whether a tile track holds one value over [first, last]: a flat line whose
// point is due at `first`, so every frame adds the same +0 or -0 to its value.
__device__ __forceinline__ bool tileTrackFixed(const TileTrack& t, int first)
{
    return t.frame != INT_MIN && t.step == 0.f && first >= t.frame;
}

// A tile's voice as the mix reads it (the staged and unstaged paths alike).
__device__ __forceinline__ MixVoice mixVoiceOf(const BatchView& b, const SegmentView& s, int index)
{
    const cs_voice_span& v = b.voices[index];
    MixVoice m;
    m.begin = v.begin;
    m.end = v.end;
    m.index = index;
    m.sharedEnd = 0;
    m.gainLeft = m.gainRight = 0.f;
    m.piece = kPieceAny;
    if (v.filterTrack >= 0) {
        m.kind = v.channels == 1 ? 2 : 1;
        m.offset = (long long)s.scratchOffset[index] - (long long)max(v.begin, s.first) * v.channels;
    } else {
        m.kind = 0;
        m.offset = 0;
        if (b.sharedRefs) {
            const SharedRef ref = b.sharedRefs[index];
            if (ref.offset >= 0) {
                m.kind = v.channels == 1 ? 3 : 4;
                m.offset = ref.offset - (long long)v.begin * v.channels;
                m.sharedEnd = v.begin + ref.frames;
            }
        }
    }
    return m;
}

constexpr int kMixStaged = kMixThreads / kTilesPerBlock;     // staged voices per tile

// Inline: 1 when some unfiltered voice is resampled by the mix itself (the
// general kernel, given more registers for the resampler); 2 when every unfiltered
// voice reads a shared source; 0 when every voice is filtered.  The lighter
// kernels keep 64 warps resident.
//
// Per tile the CTA stages, before any frame is mixed, the voice list (range,
// kind, sample offset) and the job's three control tracks (TileTrack), and for
// shared-source voices without modulation or stereo matrix under a fixed pan,
// their pan gains: a frame then reads its voice's envelope and source and two
// staged gains instead of walking bindings and evaluating pan gains, and looks up
// no track point where the tile sits on one line of each track.  Every value is
// the one the per-frame expressions give, so the sums are unchanged.
// Part 0 mixes any block; Part 1 mixes only blocks of unmodulated shared-source
// voices (the four-frame path) and appends the others to `deferred` (a count,
// then block indices); Part 2 mixes a deferred block.  Splitting keeps the lean
// pass free of the general path's registers.
template <bool Natural, int Inline, int Part>
__device__ __forceinline__ void mixBlock(const BatchView& b, const SegmentView& s, StereoStats* stats, int block,
                                         int* deferred)
{
    __shared__ double reduceD[32];
    __shared__ float reduceF[32];
    // The four tiles' voice lists, staged once for the block's 1024 frames, so a
    // frame's walk over its voices reads shared memory and then the voice's samples.
    __shared__ MixVoice staged[kTilesPerBlock][kMixStaged];
    __shared__ MixTile tiles[kTilesPerBlock];
    __shared__ TileTrack tracks[kTilesPerBlock][3];     // CC7, CC11, pan
    // Per warp: bit k of mixed / general marks tile k as not all staged stereo
    // filtered voices / not all staged kind 5 / 6 voices.
    __shared__ unsigned warpFlags[kMixThreads / 32][2];
    const int jobIndex = b.blockJob[block];
    const JobInfo job = b.jobs[jobIndex];
    const int local = block - job.blockFirst;
    const int jobTiles = (job.frames + kTileFrames - 1) / kTileFrames;
    // Tile k's three tracks are staged by threads 32-34 of its group of kMixStaged
    // threads: a warp whose first lanes stage voices (a tile rarely holds more than
    // 32), so the track lookups and the voice staging run in different warps instead
    // of one after the other in the same one.
    static_assert(kMixStaged == 64 && kTilesPerBlock * kMixStaged == kMixThreads, "one 64-thread group per tile");
    if ((threadIdx.x & 63) >= 32 && (threadIdx.x & 63) < 35) {
        const int k = int(threadIdx.x) >> 6, track = int(threadIdx.x & 63) - 32;
        const int first = local * kBlockFrames + k * kTileFrames;
        const int last = min(first + kTileFrames, max(job.frames, first + 1)) - 1;
        tracks[k][track] = tileTrackOf(b.points, job.tracks[track], job.tracks[track + 1], first, last);
    }
    {
        const int k = int(threadIdx.x) / kMixStaged, i = int(threadIdx.x) % kMixStaged;
        const int tileIndex = local * kTilesPerBlock + k;
        const MixTile tile = tileIndex < jobTiles ? b.tiles[job.tileFirst + tileIndex] : MixTile{0, 0};
        unsigned mixed = 0, general = 0;
        if (i == 0) {
            tiles[k] = tile;
            if (tile.count > kMixStaged)
                mixed = general = 1u << k;
        }
        if (i < tile.count && tile.count <= kMixStaged) {
            const int first = local * kBlockFrames + k * kTileFrames;
            // The tile's pan track, as the track staging above finds it; looked up
            // before the voice so that its loads and the voice's overlap.
            const TileTrack pan = tileTrackOf(b.points, job.tracks[2], job.tracks[3], first,
                                              min(first + kTileFrames, max(job.frames, first + 1)) - 1);
            MixVoice m = mixVoiceOf(b, s, __ldg(b.indices + tile.first + i));
            if (m.kind != 1)
                mixed |= 1u << k;
            if (m.kind >= 3) {
                const cs_voice_span& v = b.voices[m.index];
                if (v.modulationCount == 0 && !v.stereoMatrix && tileTrackFixed(pan, first)) {
                    // voiceOutputFrom with no bindings: the pan offset is the track's.
                    const float2 gains = panGains(v, fmaf(pan.step, float(first - pan.frame), pan.value));
                    m.gainLeft = gains.x;
                    m.gainRight = gains.y;
                    m.kind += 2;
                    const int last = min(first + kTileFrames, max(job.frames, first + 1)) - 1;
                    stageEnvelope(m, v, max(first, m.begin), min(last, m.end - 1));
                }
            }
            if (m.kind < 5)
                general |= 1u << k;
            staged[k][i] = m;
        }
        mixed = __reduce_or_sync(0xffffffffu, mixed);
        general = __reduce_or_sync(0xffffffffu, general);
        if ((threadIdx.x & 31) == 0) {
            warpFlags[threadIdx.x >> 5][0] = mixed;
            warpFlags[threadIdx.x >> 5][1] = general;
        }
    }
    __syncthreads();
    unsigned mixedTiles = 0, generalTiles = 0;
    #pragma unroll
    for (int w = 0; w < kMixThreads / 32; ++w) {
        mixedTiles |= warpFlags[w][0];
        generalTiles |= warpFlags[w][1];
    }
    if (Part == 1 && generalTiles != 0) {
        if (threadIdx.x == 0)
            deferred[1 + atomicAdd(deferred, 1)] = block;
        return;
    }
    double power = 0;
    float peak = 0;
    if (Inline == 2 && generalTiles == 0) {
        // Every voice of the block is an unmodulated shared-source voice under a
        // fixed pan: each thread takes four consecutive frames of one tile and
        // reads each voice's fields once for them (the voices still reach every
        // frame in span order).
        const int k = int(threadIdx.x) / (kTileFrames / 4);
        const int first = local * kBlockFrames + k * kTileFrames + (int(threadIdx.x) % (kTileFrames / 4)) * 4;
        const MixTile tile = tiles[k];
        float left[4] = {0.f, 0.f, 0.f, 0.f}, right[4] = {0.f, 0.f, 0.f, 0.f};
        for (int i = 0; i < tile.count; ++i) {
            const MixVoice& m = staged[k][i];
            if (first + 3 < m.begin || first >= m.end)
                continue;
            #pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int frame = first + j;
                if (frame < m.begin || frame >= m.end)
                    continue;
                const float level = envelopeOf(m, b.voices, frame);
                if (level > 0) {
                    float2 source = make_float2(0.f, 0.f);
                    if (frame < m.sharedEnd) {
                        if (m.kind == 5) {
                            const float x = __ldg(b.shared + (m.offset + frame));
                            source = make_float2(x, x);
                        } else {
                            source = __ldg(reinterpret_cast<const float2*>(b.shared + (m.offset + 2ll * frame)));
                        }
                    }
                    // As voiceOutputFrom: each product rounded before the sum.
                    left[j] += __fmul_rn(source.x * m.gainLeft, level);
                    right[j] += __fmul_rn(source.y * m.gainRight, level);
                }
            }
        }
        #pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int frame = first + j;
            if (frame >= job.frames || frame < s.first || frame >= s.end)
                continue;
            const float amplitude = tileTrackAt(tracks[k][0], b.points, frame) * tileTrackAt(tracks[k][1], b.points, frame);
            const float x = fmaf(left[j], amplitude, 0.f), y = fmaf(right[j], amplitude, 0.f);
            if (Natural) {
                static_cast<float2*>(b.mix)[job.offset + frame] = make_float2(x, y);
                if (!isfinite(x) || !isfinite(y)) {
                    peak = __int_as_float(0x7f800000);
                } else {
                    peak = fmaxf(peak, fmaxf(fabsf(x), fabsf(y)));
                    power += double(__fmul_rn(x, x)) + double(__fmul_rn(y, y));
                }
            } else {
                static_cast<short2*>(b.mix)[job.offset + frame] = make_short2(toPcm16(x), toPcm16(y));
            }
        }
    } else if (Part != 1)
    for (int k = 0; k < kTilesPerBlock; ++k) {
        const int frame = local * kBlockFrames + k * kTileFrames + int(threadIdx.x);
        if (frame >= job.frames || frame < s.first || frame >= s.end)
            continue;
        const MixTile tile = tiles[k];
        const float pan = tileTrackAt(tracks[k][2], b.points, frame);
        float left = 0, right = 0, wetLeft = 0, wetRight = 0;
        const auto addVoice = [&](const MixVoice& m) {
            if (frame < m.begin || frame >= m.end)
                return;
            if (m.kind == 1) {
                const float2 sample = *reinterpret_cast<const float2*>(b.filtered + (m.offset + 2ll * frame));
                wetLeft += sample.x;
                wetRight += sample.y;
            } else if (m.kind == 2) {
                // Mono filtered voices are panned after the filter.
                const cs_voice_span& v = b.voices[m.index];
                const float x = b.filtered[m.offset + frame];
                float offset = pan;
                for (int j = v.firstModulation; j < v.firstModulation + v.modulationCount; ++j) {
                    const cs_voice_modulation mod = b.modulation[j];
                    if (mod.target == CS_MOD_PAN)
                        offset += bindingAt(mod, b.points, frame);
                }
                const float2 gains = panGains(v, offset);
                wetLeft += x * gains.x;
                wetRight += x * gains.y;
            } else if (Inline == 1 && m.kind == 0) {
                const float2 sample = voiceFrame<true>(b.bank, b.sinc, b.voices[m.index], b.points, b.modulation,
                                                       pan, frame, false, -1.0);
                left += sample.x;
                right += sample.y;
            } else if (Inline && m.kind >= 5) {
                // voiceFrame with no bindings, its source read from the shared
                // sources and its pan gains and envelope piece staged for the tile.
                const float level = envelopeOf(m, b.voices, frame);
                if (level > 0) {
                    float2 source = make_float2(0.f, 0.f);
                    if (frame < m.sharedEnd) {
                        if (m.kind == 5) {
                            const float x = __ldg(b.shared + (m.offset + frame));
                            source = make_float2(x, x);
                        } else {
                            source = __ldg(reinterpret_cast<const float2*>(b.shared + (m.offset + 2ll * frame)));
                        }
                    }
                    // voiceOutputFrom rounds each product before the sum (its
                    // result joins other paths), so no multiply-add is fused here.
                    const float l = source.x * m.gainLeft;
                    const float r = source.y * m.gainRight;
                    left += __fmul_rn(l, level);
                    right += __fmul_rn(r, level);
                }
            } else if (Inline && m.kind >= 3) {
                // voiceFrame with the source read from the shared sources.
                const cs_voice_span& v = b.voices[m.index];
                const float level = envelopeAt(v, frame);
                if (level > 0) {
                    const VoiceMods mods = voiceMods(v, b.points, b.modulation, level, pan, frame);
                    float2 source = make_float2(0.f, 0.f);
                    if (frame < m.sharedEnd) {
                        if (m.kind == 3) {
                            const float x = __ldg(b.shared + (m.offset + frame));
                            source = make_float2(x, x);
                        } else {
                            source = __ldg(reinterpret_cast<const float2*>(b.shared + (m.offset + 2ll * frame)));
                        }
                    }
                    const float2 sample = voiceOutputFrom(source, v, mods, false);
                    left += sample.x;
                    right += sample.y;
                }
            }
        };
        if (!(mixedTiles >> k & 1)) {
            // Stereo filtered voices only: four voices' frames loaded at a time, then
            // added in span order, so more loads are in flight per thread.
            int i = 0;
            for (; i + 4 <= tile.count; i += 4) {
                float2 sample[4];
                bool live[4];
                #pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const MixVoice& m = staged[k][i + u];
                    live[u] = frame >= m.begin && frame < m.end;
                    sample[u] = live[u] ? *reinterpret_cast<const float2*>(b.filtered + (m.offset + 2ll * frame))
                                        : make_float2(0.f, 0.f);
                }
                #pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (live[u]) {
                        wetLeft += sample[u].x;
                        wetRight += sample[u].y;
                    }
            }
            for (; i < tile.count; ++i)
                addVoice(staged[k][i]);
        } else if (tile.count <= kMixStaged) {
            for (int i = 0; i < tile.count; ++i)
                addVoice(staged[k][i]);
        } else {
            for (int i = tile.first; i < tile.first + tile.count; ++i)
                addVoice(mixVoiceOf(b, s, __ldg(b.indices + i)));
        }
        // CC7 x CC11 (jobGainAt).
        const float amplitude = tileTrackAt(tracks[k][0], b.points, frame) * tileTrackAt(tracks[k][1], b.points, frame);
        const float x = fmaf(left, amplitude, wetLeft), y = fmaf(right, amplitude, wetRight);
        if (Natural) {
            static_cast<float2*>(b.mix)[job.offset + frame] = make_float2(x, y);
            if (!isfinite(x) || !isfinite(y)) {
                peak = __int_as_float(0x7f800000);
            } else {
                peak = fmaxf(peak, fmaxf(fabsf(x), fabsf(y)));
                power += double(__fmul_rn(x, x)) + double(__fmul_rn(y, y));
            }
        } else {
            static_cast<short2*>(b.mix)[job.offset + frame] = make_short2(toPcm16(x), toPcm16(y));
        }
    }
    if (Natural) {
        blockStats(power, peak, reduceD, reduceF);
        if (threadIdx.x == 0)
            stats[block] = {power, peak};
    }
}

template <bool Natural, int Inline>
__global__ void __launch_bounds__(kMixThreads, Inline == 1 ? 5 : 8) mixKernel(BatchView b, SegmentView s, StereoStats* stats)
{
    mixBlock<Natural, Inline, 0>(b, s, stats, s.blocks[blockIdx.x], nullptr);
}

template <bool Natural>
__global__ void __launch_bounds__(kMixThreads, 8) mixLeanKernel(BatchView b, SegmentView s, StereoStats* stats,
                                                                 int* deferred)
{
    mixBlock<Natural, 2, 1>(b, s, stats, s.blocks[blockIdx.x], deferred);
}

// The deferred blocks, each CTA taking every gridDim.x-th.
template <bool Natural>
__global__ void __launch_bounds__(kMixThreads, 8) mixDeferredKernel(BatchView b, SegmentView s, StereoStats* stats,
                                                                     const int* deferred)
{
    const int count = deferred[0];
    for (int i = int(blockIdx.x); i < count; i += int(gridDim.x)) {
        mixBlock<Natural, 2, 2>(b, s, stats, deferred[1 + i], nullptr);
        __syncthreads();                // the next block restages the shared arrays
    }
}

// Power and peak of each 1024-frame block of an existing float mix (the block scan
// that mixKernel fuses into synthesis, for a mix produced elsewhere).
__global__ void __launch_bounds__(kMixThreads) scanKernel(BatchView b, StereoStats* stats, int blocks)
{
    __shared__ double reduceD[32];
    __shared__ float reduceF[32];
    const int block = int(blockIdx.x);
    if (block >= blocks)
        return;
    const JobInfo job = b.jobs[b.blockJob[block]];
    const int first = (block - job.blockFirst) * kBlockFrames;
    const int end = min(first + kBlockFrames, job.frames);
    const float2* mix = static_cast<const float2*>(b.mix) + job.offset;
    double power = 0;
    float peak = 0;
    for (int frame = first + int(threadIdx.x); frame < end; frame += blockDim.x) {
        const float2 v = mix[frame];
        if (!isfinite(v.x) || !isfinite(v.y)) {
            peak = __int_as_float(0x7f800000);
        } else {
            peak = fmaxf(peak, fmaxf(fabsf(v.x), fabsf(v.y)));
            power += double(__fmul_rn(v.x, v.x)) + double(__fmul_rn(v.y, v.y));
        }
    }
    blockStats(power, peak, reduceD, reduceF);
    if (threadIdx.x == 0)
        stats[block] = {power, peak};
}

// ---- finishing (src/cuda/tail.cu) ------------------------------------------------------

// ---- natural endpoint, peak repair and scale (tail.cu:83-139) -------------------------
//
// The reference walks each job's 1024-frame blocks in order on one thread: the
// first block at or after the music's end whose power is at most 1e-12 per sample
// (re-summed in frame order near the threshold), or the first non-finite block,
// ends the search, and the peak is the loudest block before it (and the quiet
// block itself).  Here every block is tested at once: the first stopping block is
// an integer minimum (atomicMin), the peak an integer maximum of the non-negative
// float bits (atomicMax), so the result is the walk's whatever the order; a thread
// per job then applies the end rules.

__global__ void scanResetKernel(FinishView f, int jobs)
{
    const int j = int(blockIdx.x * blockDim.x + threadIdx.x);
    if (j < jobs)
        f.scans[j] = JobScan{INT_MAX, 0, -1, 0, 0ull};
}

// Thread per block: does the block stop the natural search, and how.
__global__ void nativeStopKernel(BatchView b, FinishView f, int blocks)
{
    const int g = int(blockIdx.x * blockDim.x + threadIdx.x);
    if (g >= blocks)
        return;
    const int jobIndex = b.blockJob[g];
    const JobInfo job = b.jobs[jobIndex];
    const int block = g - job.blockFirst;
    const StereoStats stat = f.stereo[g];
    const bool bad = !isfinite(stat.peak);
    const int first = block * kBlockFrames;
    const int blockEnd = min(job.limit, first + kBlockFrames);
    bool quiet = false;
    if (!bad && blockEnd >= job.musicEnd) {
        const double threshold = 1e-12 * (blockEnd - first) * 2;
        double power = stat.power;
        // Near the threshold, re-sum in frame order as the host does.
        if (fabs(power - threshold) <= threshold * 1e-12) {
            power = 0;
            const float2* mix = static_cast<const float2*>(b.mix) + job.offset;
            for (int frame = first; frame < min(blockEnd, job.frames); ++frame) {
                const float2 value = mix[frame];
                power += __fmul_rn(value.x, value.x);
                power += __fmul_rn(value.y, value.y);
            }
        }
        quiet = power <= threshold;
    }
    if (bad || quiet)
        atomicMin(&f.scans[jobIndex].stop, 2 * block + (bad ? 1 : 0));
}

// Thread per block: the peak over the blocks the walk reads before stopping.
__global__ void nativePeakKernel(BatchView b, FinishView f, int blocks)
{
    const int g = int(blockIdx.x * blockDim.x + threadIdx.x);
    if (g >= blocks)
        return;
    const int jobIndex = b.blockJob[g];
    const int block = g - b.jobs[jobIndex].blockFirst;
    const int stop = f.scans[jobIndex].stop;
    const int stopBlock = stop == INT_MAX ? INT_MAX : stop >> 1;
    if (block < stopBlock || (block == stopBlock && !(stop & 1))) {
        const float peak = f.stereo[g].peak;           // finite and >= 0 here
        if (peak > 0)
            atomicMax(&f.scans[jobIndex].peak, __float_as_int(peak));
    }
}

// Thread per job: status, end frame, data frames and scale.
__global__ void nativeResultKernel(BatchView b, FinishView f)
{
    const int jobIndex = int(blockIdx.x * blockDim.x + threadIdx.x);
    if (jobIndex >= b.jobCount)
        return;
    const JobInfo job = b.jobs[jobIndex];
    const JobScan scan = f.scans[jobIndex];
    cs_tail_result result{};
    int end = 0;
    if (scan.stop != INT_MAX) {
        if (scan.stop & 1) {
            result.status = CS_TAIL_NONFINITE;
            f.results[jobIndex] = result;
            return;
        }
        end = min(job.limit, (scan.stop >> 1) * kBlockFrames + kBlockFrames);
    }
    const float peak = __int_as_float(scan.peak);
    if (!end) {
        const int silent = (job.frames + kBlockFrames - 1) / kBlockFrames * kBlockFrames;
        if (silent < job.limit)
            end = min(job.limit, max(silent + kBlockFrames,
                                     (job.musicEnd + kBlockFrames - 1) / kBlockFrames * kBlockFrames));
    }
    if (!end) {
        result.status = CS_TAIL_DURATION;
    } else {
        const double attenuation = peak >= 1 ? 20 * log10(double(peak)) + 1 : 0;
        if (attenuation > 5 + 1e-6) {
            result.status = CS_TAIL_PEAK;
        } else {
            result.frames = end;
            result.dataFrames = min(end, job.frames);
            result.scale = float(32768 * pow(10., -attenuation / 20));
        }
    }
    f.results[jobIndex] = result;
}

// Warps per CTA of the warp-per-unit finishing kernels, and a warp-wide reduction.
constexpr int kFinalizeWarps = 8;

template <class T, class Op>
__device__ __forceinline__ T warpAll(T value, Op op)
{
    #pragma unroll
    for (int d = 16; d; d >>= 1)
        value = op(value, __shfl_xor_sync(0xffffffffu, value, d));
    return value;
}

// Mono PCM16 with ties-to-even channel average and per-window stats (tail.cu:147-181).
// A warp per 50 ms window (eight per CTA).  The window's power is a sum of squared
// 16-bit integers, below 2^53, so every partial sum is exact and any order gives
// the reference's double.
__global__ void __launch_bounds__(kFinalizeWarps * 32) quantizeMonoKernel(BatchView b, FinishView f, int window)
{
    const int w = int(blockIdx.x) * kFinalizeWarps + int(threadIdx.x >> 5);
    const int lane = int(threadIdx.x & 31);
    if (w >= f.windowCount)
        return;
    const int jobIndex = b.windowJob[w];
    const JobInfo job = b.jobs[jobIndex];
    const cs_tail_result& result = f.results[jobIndex];
    const int first = (w - job.windowFirst) * window;
    const int end = min(first + window, result.dataFrames);
    if (first >= end)
        return;
    const float scale = result.scale;
    const float2* __restrict__ mix = static_cast<const float2*>(b.mix) + job.offset;
    short* __restrict__ mono = f.mono + job.offset;
    double power = 0;
    int peak = 0;
    // Each lane takes kUnroll frames 32 apart per step, their loads issued together.
    constexpr int kUnroll = 4;
    for (int base = first + lane; base < end; base += 32 * kUnroll) {
        float2 sample[kUnroll];
        #pragma unroll
        for (int u = 0; u < kUnroll; ++u)
            sample[u] = base + 32 * u < end ? __ldcs(mix + base + 32 * u) : make_float2(0.f, 0.f);
        #pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            const int frame = base + 32 * u;
            if (frame >= end)
                break;
            const int left = __float2int_rn(fminf(32767.f, fmaxf(-32768.f, sample[u].x * scale)));
            const int right = __float2int_rn(fminf(32767.f, fmaxf(-32768.f, sample[u].y * scale)));
            const int sum = left + right;
            const int value = (sum >> 1) + ((sum & 1) & ((sum >> 1) & 1));
            mono[frame] = short(value);
            power += double(value) * value;
            peak = max(peak, abs(value));
        }
    }
    power = warpAll(power, SumOp{});
    peak = warpAll(peak, MaxOp{});
    if (lane == 0)
        f.windows[w] = {power, peak};
}

// ---- weak-tail trim (tail.cu:183-213) ---------------------------------------------------
//
// The threshold follows from the loudest 50 ms window of the job's PCM (an integer
// maximum of the non-negative double bits) and the trim point from the last
// window above it (an integer maximum of window indices), each window tested by
// its own thread; a thread per job applies the trim.

__device__ __forceinline__ bool trimWindow(const BatchView& b, const FinishView& f, int w, int& jobIndex, int& index)
{
    jobIndex = b.windowJob[w];
    if (f.results[jobIndex].status != CS_TAIL_OK)
        return false;
    index = w - b.jobs[jobIndex].windowFirst;
    return index < 0 ? false : true;
}

__global__ void trimPowerKernel(BatchView b, FinishView f, TailConfig config, int windows)
{
    const int w = int(blockIdx.x * blockDim.x + threadIdx.x);
    int jobIndex, index;
    if (w >= windows || !trimWindow(b, f, w, jobIndex, index))
        return;
    const int count = (f.results[jobIndex].dataFrames + config.window - 1) / config.window;
    if (index < count)
        atomicMax(&f.scans[jobIndex].maxPower, (unsigned long long)__double_as_longlong(f.windows[w].power));
}

__global__ void trimLastKernel(BatchView b, FinishView f, TailConfig config, int windows)
{
    const int w = int(blockIdx.x * blockDim.x + threadIdx.x);
    int jobIndex, index;
    if (w >= windows || !trimWindow(b, f, w, jobIndex, index))
        return;
    const int count = (f.results[jobIndex].dataFrames + config.window - 1) / config.window;
    if (index >= count)
        return;
    const double maxPower = __longlong_as_double((long long)f.scans[jobIndex].maxPower);
    const double threshold = fmin(config.ceiling, fmax(config.floor, sqrt(maxPower / config.window) * config.relative));
    const MonoStats stat = f.windows[w];
    if (sqrt(stat.power / config.window) > threshold || stat.peak > threshold * 4)
        atomicMax(&f.scans[jobIndex].last, index);
}

__global__ void trimResultKernel(BatchView b, FinishView f, TailConfig config)
{
    const int jobIndex = int(blockIdx.x * blockDim.x + threadIdx.x);
    if (jobIndex >= b.jobCount)
        return;
    cs_tail_result& result = f.results[jobIndex];
    const int last = f.scans[jobIndex].last;
    if (result.status != CS_TAIL_OK || last < 0)
        return;
    const int lastSound = min(result.frames, (last + 1) * config.window);
    if (result.frames - lastSound >= config.quietFrames) {
        result.frames = lastSound + config.padding;
        result.dataFrames = min(result.frames, result.dataFrames);
        result.fade = min(result.frames, config.fade);
    }
}

// Output offsets: exclusive prefix of dataFrames over jobs in plan order
// (tail.cu:216-238), one warp.
__global__ void layoutKernel(BatchView b, FinishView f, int natural)
{
    const int lane = int(threadIdx.x);
    unsigned long long carry = 0;
    for (int base = 0; base < b.jobCount; base += 32) {
        const int i = base + lane;
        unsigned long long own = 0;
        if (i < b.jobCount) {
            cs_tail_result& result = f.results[i];
            if (!natural) {
                const JobInfo job = b.jobs[i];
                result = cs_tail_result{};
                result.frames = job.frames;
                result.dataFrames = job.frames;
                result.fade = job.fade;
            }
            own = (unsigned long long)result.dataFrames;
        }
        unsigned long long scan = own;
        #pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const unsigned long long up = __shfl_up_sync(0xffffffffu, scan, d);
            if (lane >= d) scan += up;
        }
        if (i < b.jobCount) {
            cs_tail_result& result = f.results[i];
            result.offset = carry + scan - own;
            result.peak = 0;
            result.first = result.frames;
            result.last = -1;
        }
        carry += __shfl_sync(0xffffffffu, scan, 31);
    }
}

// Out of line: only the last frames of a job fade, and the FP64 cosine would
// otherwise hold registers through the whole finishing loop.
__device__ __noinline__ short fadeSample(short value, int index, int count)
{
    constexpr double pi = 3.14159265358979323846;
    const double gain = count == 1 ? 0 : .5 * (1 + cos(pi * index / (count - 1)));
    return short(__double2int_rn(value * gain));
}

// Fade, compaction and peak / audible range (tail.cu:240-297).  When the quality
// gate or group volume is on, the same pass sums the mono power of the samples it
// writes into the job's 250 ms body windows (measureBody, quality.cu:21-39): the
// sums are integers, so the warp partials and atomics give the reference's
// totals in any order.  A warp per 1024-frame block (eight per CTA), each lane
// every 32nd frame; the reductions are warp shuffles, so no CTA barrier is needed.
template <int Channels, bool Assess>
__global__ void __launch_bounds__(kFinalizeWarps * 32, 4) finalizeKernel(BatchView b, FinishView f, const short* input,
                                                                      int quality)
{
    const int block = int(blockIdx.x) * kFinalizeWarps + int(threadIdx.x >> 5);
    const int lane = int(threadIdx.x & 31);
    if (block >= f.blockCount)
        return;
    const int jobIndex = b.blockJob[block];
    const JobInfo job = b.jobs[jobIndex];
    cs_tail_result& result = f.results[jobIndex];
    const uint64_t outputOffset = result.offset;
    const int frames = result.frames, fade = result.fade;
    const int first = (block - job.blockFirst) * kBlockFrames;
    const int end = min(first + kBlockFrames, result.dataFrames);
    if (first >= end)
        return;
    // Body windows this block touches: [windowA, windowB]; frames before `split`
    // belong to windowA.
    int bodyEnd = 0, windowA = 0, windowB = 0, split = 0, bodyFirst = 0;
    if (Assess && f.bodyPower && result.status == CS_TAIL_OK) {
        const AssessJob a = f.assess[jobIndex];
        bodyEnd = min(a.bodyFrames, end);
        bodyFirst = a.bodyFirst;
        if (first < bodyEnd) {
            windowA = f.body.windowOf(first);
            windowB = f.body.windowOf(bodyEnd - 1);
            split = f.body.start(windowA + 1);
        }
    }
    const bool paired = windowB - windowA <= 1;
    unsigned long long powerA = 0, powerB = 0;
    int peak = 0, audibleFirst = frames, audibleLast = -1, clipped = 0;
    const int fadeStart = frames - fade;
    const short* __restrict__ source = input + job.offset * Channels;
    short* __restrict__ packed = f.packed + outputOffset * Channels;
    // Each lane takes kUnroll frames 32 apart per step, their loads issued together:
    // sixteen 2-byte loads in flight per lane (four CTAs per SM) keep enough bytes
    // in flight to hide DRAM latency, which four did not (0.935 against 0.975 ms on
    // a 293 M-frame batch).
    constexpr int kUnroll = 16;
    for (int base = first + lane; base < end; base += 32 * kUnroll) {
        short loaded[kUnroll][Channels];
        #pragma unroll
        for (int u = 0; u < kUnroll; ++u)
            #pragma unroll
            for (int c = 0; c < Channels; ++c)
                loaded[u][c] = base + 32 * u < end ? __ldcs(source + (base + 32 * u) * Channels + c) : short(0);
        #pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            const int frame = base + 32 * u;
            if (frame >= end)
                break;
            int framePeak = 0, mono = 0;
            #pragma unroll
            for (int c = 0; c < Channels; ++c) {
                short value = loaded[u][c];
                if (frame >= fadeStart)
                    value = fadeSample(value, frame - fadeStart, fade);
                packed[frame * Channels + c] = value;
                const int magnitude = abs(int(value));
                framePeak = max(framePeak, magnitude);
                if (Assess)
                clipped += magnitude >= 32767;
                mono += Channels == 1 ? 2 * int(value) : int(value);
            }
            peak = max(peak, framePeak);
            if (framePeak > 3) {
                audibleFirst = min(audibleFirst, frame);
                audibleLast = frame;
            }
            if (Assess && frame < bodyEnd) {
                const unsigned long long power = (unsigned long long)((long long)mono * mono);
                if (!paired)
                    atomicAdd(f.bodyPower + bodyFirst + f.body.windowOf(frame), power);
                else if (frame < split)
                    powerA += power;
                else
                    powerB += power;
            }
        }
    }
    peak = warpAll(peak, MaxOp{});
    audibleFirst = warpAll(audibleFirst, MinOp{});
    audibleLast = warpAll(audibleLast, MaxOp{});
    if (Assess)
        clipped = warpAll(clipped, SumOp{});
    if (Assess && first < bodyEnd && paired) {
        powerA = warpAll(powerA, SumOp{});
        powerB = warpAll(powerB, SumOp{});
        if (lane == 0) {
            atomicAdd(f.bodyPower + bodyFirst + windowA, powerA);
            if (windowB != windowA)
                atomicAdd(f.bodyPower + bodyFirst + windowB, powerB);
        }
    }
    if (lane == 0) {
        if (Assess && quality && clipped)
            atomicAdd(&result.audio.clipped, clipped);
        if (audibleLast >= 0) {
            atomicMax(&result.peak, peak);
            atomicMin(&result.first, audibleFirst);
            atomicMax(&result.last, audibleLast);
        }
    }
}

// ---- mix tile voice lists ---------------------------------------------------------------
//
// The voice list of a 256-frame tile holds the job's spans that overlap it, in
// span order (the reference's BatchIndex::append, src/cuda/renderer.cpp:390-460).
// A CTA per (job, chunk of kIndexChunkTiles tiles).  The CTA first gathers, in
// span order, the job's spans that overlap the chunk into shared memory (an
// order-keeping compaction per 256 spans) and sums the entries of the job's
// earlier chunks; then each thread owns eight consecutive tiles of the chunk and
// walks the gathered spans in order twice, to count its tiles' voices and to
// write their lists, so each list comes out in span order and no two threads
// write the same slot.  A chunk overlapped by more spans than the shared list
// holds walks the job's spans in global memory instead.
constexpr int kIndexThreads = kIndexChunkTiles / 8;
constexpr int kIndexList = 2048;

__global__ void __launch_bounds__(kIndexThreads) tileIndexKernel(BatchView b, const JobSpans* __restrict__ spans,
                                                                 const int2* __restrict__ units, MixTile* tiles,
                                                                 int* indices)
{
    __shared__ int listSpan[kIndexList], listFirst[kIndexList], listLast[kIndexList];
    __shared__ int warpCount[kIndexThreads / 32], warpSum[kIndexThreads / 32];
    __shared__ int listed;
    const int2 unit = units[blockIdx.x];
    const JobInfo job = b.jobs[unit.x];
    const JobSpans js = spans[unit.x];
    const int jobTiles = (job.frames + kTileFrames - 1) / kTileFrames;
    const int chunkFirst = unit.y * kIndexChunkTiles, chunkLast = chunkFirst + kIndexChunkTiles - 1;
    const int lane = int(threadIdx.x & 31), warp = int(threadIdx.x >> 5);
    if (threadIdx.x == 0)
        listed = 0;
    __syncthreads();
    int before = 0;                     // entries below the chunk of this thread's spans
    for (int round = 0; round < js.voiceCount; round += kIndexThreads) {
        const int k = round + int(threadIdx.x);
        int a = 0, e = -1;
        if (k < js.voiceCount) {
            const cs_voice_span& v = b.voices[js.voiceFirst + k];
            a = v.begin / kTileFrames;
            e = (v.end - 1) / kTileFrames;
            before += max(0, min(e, chunkFirst - 1) - a + 1);
        }
        const bool overlaps = k < js.voiceCount && e >= chunkFirst && a <= chunkLast;
        const unsigned ballot = __ballot_sync(0xffffffffu, overlaps);
        if (lane == 0)
            warpCount[warp] = __popc(ballot);
        __syncthreads();
        int at = listed + __popc(ballot & ((1u << lane) - 1));
        for (int w = 0; w < warp; ++w)
            at += warpCount[w];
        if (overlaps && at < kIndexList) {
            listSpan[at] = k;
            listFirst[at] = a;
            listLast[at] = e;
        }
        __syncthreads();
        if (threadIdx.x == 0)
            for (int w = 0; w < kIndexThreads / 32; ++w)
                listed += warpCount[w];
        __syncthreads();
    }
    const bool inShared = listed <= kIndexList;
    const int candidates = inShared ? listed : js.voiceCount;
    const auto spanAt = [&](int i, int& k, int& a, int& e) {
        if (inShared) {
            k = listSpan[i];
            a = listFirst[i];
            e = listLast[i];
        } else {
            const cs_voice_span& v = b.voices[js.voiceFirst + i];
            k = i;
            a = v.begin / kTileFrames;
            e = (v.end - 1) / kTileFrames;
        }
    };
    const int first = chunkFirst + int(threadIdx.x) * 8;       // this thread's first tile
    int count[8] = {};
    for (int i = 0; i < candidates; ++i) {
        int k, a, e;
        spanAt(i, k, a, e);
        #pragma unroll
        for (int j = 0; j < 8; ++j)
            count[j] += first + j >= a && first + j <= e;
    }
    int own = 0;
    #pragma unroll
    for (int j = 0; j < 8; ++j)
        own += count[j];
    // Exclusive scan of the threads' entries in tile order, and the sum of `before`.
    int inclusive = own, total = before;
    #pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int up = __shfl_up_sync(0xffffffffu, inclusive, d);
        if (lane >= d)
            inclusive += up;
        total += __shfl_xor_sync(0xffffffffu, total, d);
    }
    if (lane == 31)
        warpCount[warp] = inclusive;
    if (lane == 0)
        warpSum[warp] = total;
    __syncthreads();
    int offset = js.indexFirst + inclusive - own;
    for (int w = 0; w < kIndexThreads / 32; ++w) {
        offset += warpSum[w];
        if (w < warp)
            offset += warpCount[w];
    }
    int cursor[8];
    #pragma unroll
    for (int j = 0; j < 8; ++j) {
        cursor[j] = offset;
        if (first + j < jobTiles)
            tiles[job.tileFirst + first + j] = MixTile{offset, count[j]};
        offset += count[j];
    }
    if (!own)
        return;
    for (int i = 0; i < candidates; ++i) {
        int k, a, e;
        spanAt(i, k, a, e);
        if (e < first || a > first + 7)
            continue;
        #pragma unroll
        for (int j = 0; j < 8; ++j)
            if (first + j >= a && first + j <= e)
                indices[cursor[j]++] = js.voiceFirst + k;
    }
}

// ---- launchers --------------------------------------------------------------------------

__global__ void expandTilesKernel(const int4* runs, int count, int2* tiles)
{
    const int4 run = runs[blockIdx.x];
    const int n = (run.z - run.y + kSourceTile - 1) / kSourceTile;
    for (int k = int(threadIdx.x); k < n; k += blockDim.x)
        tiles[run.w + k] = make_int2(run.x, run.y + k * kSourceTile);
}

void launchExpandTiles(const int4* runs, int count, int2* tiles, cudaStream_t stream)
{
    if (count)
        expandTilesKernel<<<count, 128, 0, stream>>>(runs, count, tiles);
}

void launchScan(const BatchView& b, StereoStats* stats, int blocks, cudaStream_t stream)
{
    if (blocks)
        scanKernel<<<blocks, kMixThreads, 0, stream>>>(b, stats, blocks);
}


void launchPitch(const BatchView& b, const SegmentView& s, cudaStream_t stream)
{
    if (!s.pitchCount)
        return;
    pitchKernel<<<(s.pitchCount + 63) / 64, 64, 0, stream>>>(b, s);
}

// Kernel attributes belong to a device's context, so they are set once per device:
// `set` runs under the lock the first time `slot` is seen on the current device,
// and the slot is marked done only when every attribute call succeeded (a failed
// set is retried by the next launch; no launch proceeds before the set returns).
template <class Set>
static void setOncePerDevice(int slot, Set&& set)
{
    static std::mutex guard;
    static unsigned long long done[64] = {};
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= 64) {
        set();
        return;
    }
    std::lock_guard<std::mutex> lock(guard);
    const unsigned long long bit = 1ull << slot;
    if (done[device] & bit)
        return;
    if (set() == cudaSuccess)
        done[device] |= bit;
}

int launchSharedSources(const BatchView& b, const SharedSource* sources, const int2* tiles, int tileCount,
                        cudaStream_t stream)
{
    if (!tileCount)
        return 0;
    setOncePerDevice(3, [] {
        return cudaFuncSetAttribute(sharedSourceKernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    int(kSharedSincBytes));
    });
    int device = 0, sms = 0;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const long long needed = ((long long)tileCount * kSourceTile + kSharedSourceThreads - 1) / kSharedSourceThreads;
    const int grid = int(std::max<long long>(1, std::min<long long>(needed, std::max(sms, 1))));
    sharedSourceKernel<<<grid, kSharedSourceThreads, kSharedSincBytes, stream>>>(b, sources, tiles, tileCount);
    return 1;
}

static cudaError_t firstError(std::initializer_list<cudaError_t> statuses)
{
    for (const cudaError_t s : statuses)
        if (s != cudaSuccess)
            return s;
    return cudaSuccess;
}

int launchSources(const BatchView& b, const SegmentView& s, cudaStream_t stream)
{
    if (!s.sourceTileCount)
        return 0;
    setOncePerDevice(0, [] {
        return cudaFuncSetAttribute(sourceKernel, cudaFuncAttributePreferredSharedMemoryCarveout, kOverlapCarveout);
    });
    sourceKernel<<<s.sourceTileCount, kSourceThreads, 0, stream>>>(b, s);
    return 1;
}

int launchRecurrences(const BatchView& b, const SegmentView& s, cudaStream_t stream)
{
    if (!s.simpleCount)
        return 0;
    constexpr int chainsPerCta = kRecWarps * kRecChains;
    constexpr int bytes = chainsPerCta * kRecChainBytes;
    setOncePerDevice(1, [] {
        return firstError({cudaFuncSetAttribute(recurrenceKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes),
                           cudaFuncSetAttribute(recurrenceKernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                                kOverlapCarveout)});
    });
    recurrenceKernel<<<(s.simpleCount + chainsPerCta - 1) / chainsPerCta, kRecThreads, bytes, stream>>>(
        b, s, b.error);
    return 1;
}

int launchGeneralChains(const BatchView& b, const SegmentView& s, cudaStream_t stream)
{
    if (!s.chainCount)
        return 0;
    chainKernel<<<(s.chainCount + kChainWarps - 1) / kChainWarps, kChainWarps * 32, 0, stream>>>(b, s);
    return 1;
}

// The inline mix kernels need about 33 KB of shared memory per SM (five CTAs); the
// rest of the SM's 256 KB goes to L1, where the 393 KB sinc table competes for room.
constexpr int kInlineMixCarveout = 20;

void launchTileIndex(const BatchView& b, const JobSpans* spans, const int2* units, int unitCount, MixTile* tiles,
                     int* indices, cudaStream_t stream)
{
    if (unitCount)
        tileIndexKernel<<<unitCount, kIndexThreads, 0, stream>>>(b, spans, units, tiles, indices);
}

int launchMix(const BatchView& b, const SegmentView& s, bool natural, StereoStats* stats, int* deferred,
              cudaStream_t stream)
{
    if (!s.blockCount)
        return 0;
    if (b.inlineVoices == 1)
        setOncePerDevice(2, [] {
            return firstError({cudaFuncSetAttribute(mixKernel<true, 1>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                                    kInlineMixCarveout),
                               cudaFuncSetAttribute(mixKernel<false, 1>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                                    kInlineMixCarveout)});
        });
    const auto launch = [&](auto kernel) { kernel<<<s.blockCount, kMixThreads, 0, stream>>>(b, s, stats); };
    if (b.inlineVoices == 1) {
        if (natural)
            launch(mixKernel<true, 1>);
        else
            launch(mixKernel<false, 1>);
        return 1;
    }
    if (!b.sharedRefs) {
        // No shared sources: every voice is filtered.
        if (natural)
            launch(mixKernel<true, 2>);
        else
            launch(mixKernel<false, 2>);
        return 1;
    }
    {
        // The lean pass over every block, then the blocks it deferred.
        int device = 0, sms = 0;
        cudaGetDevice(&device);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        const int grid = std::max(1, std::min(s.blockCount, std::max(sms, 1) * 8));
        cudaMemsetAsync(deferred, 0, sizeof(int), stream);
        if (natural) {
            mixLeanKernel<true><<<s.blockCount, kMixThreads, 0, stream>>>(b, s, stats, deferred);
            mixDeferredKernel<true><<<grid, kMixThreads, 0, stream>>>(b, s, stats, deferred);
        } else {
            mixLeanKernel<false><<<s.blockCount, kMixThreads, 0, stream>>>(b, s, stats, deferred);
            mixDeferredKernel<false><<<grid, kMixThreads, 0, stream>>>(b, s, stats, deferred);
        }
    }
    return 2;
}

int launchFinish(const BatchView& b, const FinishView& f, bool natural, bool quality, const TailConfig& tail,
                 cudaStream_t stream)
{
    int launches = 0;
    if (natural) {
        constexpr int threads = 256;
        const int jobGrid = (b.jobCount + threads - 1) / threads;
        const int blockGrid = (f.blockCount + threads - 1) / threads;
        const int windowGrid = (f.windowCount + threads - 1) / threads;
        scanResetKernel<<<jobGrid, threads, 0, stream>>>(f, b.jobCount);
        launches += 1;
        if (f.blockCount) {
            nativeStopKernel<<<blockGrid, threads, 0, stream>>>(b, f, f.blockCount);
            nativePeakKernel<<<blockGrid, threads, 0, stream>>>(b, f, f.blockCount);
            launches += 2;
        }
        nativeResultKernel<<<jobGrid, threads, 0, stream>>>(b, f);
        ++launches;
        if (f.windowCount) {
            quantizeMonoKernel<<<(f.windowCount + kFinalizeWarps - 1) / kFinalizeWarps, kFinalizeWarps * 32, 0,
                                 stream>>>(b, f, tail.window);
            trimPowerKernel<<<windowGrid, threads, 0, stream>>>(b, f, tail, f.windowCount);
            trimLastKernel<<<windowGrid, threads, 0, stream>>>(b, f, tail, f.windowCount);
            launches += 3;
        }
        trimResultKernel<<<jobGrid, threads, 0, stream>>>(b, f, tail);
        ++launches;
    }
    layoutKernel<<<1, 32, 0, stream>>>(b, f, natural ? 1 : 0);
    ++launches;
    if (f.blockCount) {
        const int grid = (f.blockCount + kFinalizeWarps - 1) / kFinalizeWarps, threads = kFinalizeWarps * 32;
        const short* pcm = natural ? f.mono : static_cast<const short*>(b.mix);
        const bool assess = quality || f.bodyPower;
        if (natural && assess)
            finalizeKernel<1, true><<<grid, threads, 0, stream>>>(b, f, pcm, quality ? 1 : 0);
        else if (natural)
            finalizeKernel<1, false><<<grid, threads, 0, stream>>>(b, f, pcm, 0);
        else if (assess)
            finalizeKernel<2, true><<<grid, threads, 0, stream>>>(b, f, pcm, quality ? 1 : 0);
        else
            finalizeKernel<2, false><<<grid, threads, 0, stream>>>(b, f, pcm, 0);
        ++launches;
    }
    return launches;
}

} // namespace cs
