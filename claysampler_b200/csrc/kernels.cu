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

#include <cmath>
#include <cstdio>

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

// ---- mix + block scan ----------------------------------------------------------------

constexpr int kMixThreads = 256;

template <class T, class Op>
__device__ __forceinline__ T blockReduce(T value, T identity, Op op, T* scratch)
{
    #pragma unroll
    for (int d = 16; d; d >>= 1)
        value = op(value, __shfl_down_sync(0xffffffffu, value, d));
    const int warp = int(threadIdx.x >> 5), lane = int(threadIdx.x & 31);
    __syncthreads();
    if (!lane)
        scratch[warp] = value;
    __syncthreads();
    if (warp == 0) {
        value = lane < int(blockDim.x >> 5) ? scratch[lane] : identity;
        #pragma unroll
        for (int d = 16; d; d >>= 1)
            value = op(value, __shfl_down_sync(0xffffffffu, value, d));
    }
    return value;                       // valid in thread 0
}

struct SumOp { template <class T> __device__ T operator()(T a, T b) const { return a + b; } };
struct MaxOp { template <class T> __device__ T operator()(T a, T b) const { return a > b ? a : b; } };
struct MinOp { __device__ int operator()(int a, int b) const { return a < b ? a : b; } };

template <bool Natural>
__global__ void __launch_bounds__(kMixThreads) mixKernel(BatchView b, SegmentView s, StereoStats* stats)
{
    __shared__ double reduceD[32];
    __shared__ float reduceF[32];
    const int block = s.blocks[blockIdx.x];
    const int jobIndex = b.blockJob[block];
    const JobInfo job = b.jobs[jobIndex];
    const int local = block - job.blockFirst;
    double power = 0;
    float peak = 0;
    for (int k = 0; k < kTilesPerBlock; ++k) {
        const int frame = local * kBlockFrames + k * kTileFrames + int(threadIdx.x);
        if (frame >= job.frames || frame < s.first || frame >= s.end)
            continue;
        const MixTile tile = b.tiles[job.tileFirst + local * kTilesPerBlock + k];
        const float pan = trackAt(b.points, job.tracks[2], job.tracks[3], frame);
        float left = 0, right = 0, wetLeft = 0, wetRight = 0;
        for (int i = tile.first; i < tile.first + tile.count; ++i) {
            const int index = __ldg(b.indices + i);
            const cs_voice_span& v = b.voices[index];
            if (frame < v.begin || frame >= v.end)
                continue;
            if (v.filterTrack >= 0) {
                const float* src = b.filtered + s.scratchOffset[index] + size_t(frame - max(v.begin, s.first)) *
                    v.channels;
                float2 sample = make_float2(src[0], v.channels == 1 ? src[0] : src[1]);
                if (v.channels == 1) {
                    float offset = pan;
                    for (int j = v.firstModulation; j < v.firstModulation + v.modulationCount; ++j) {
                        const cs_voice_modulation m = b.modulation[j];
                        if (m.target == CS_MOD_PAN)
                            offset += bindingAt(m, b.points, frame);
                    }
                    const float2 gains = panGains(v, offset);
                    sample.x *= gains.x;
                    sample.y *= gains.y;
                }
                wetLeft += sample.x;
                wetRight += sample.y;
            } else {
                const float2 sample = voiceFrame(b.bank, b.sinc, v, b.points, b.modulation, pan, frame, false, -1.0);
                left += sample.x;
                right += sample.y;
            }
        }
        const float amplitude = jobGainAt(b.points, job.tracks, frame);
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
        power = blockReduce(power, 0.0, SumOp{}, reduceD);
        peak = blockReduce(peak, 0.f, MaxOp{}, reduceF);
        if (threadIdx.x == 0)
            stats[block] = {power, peak};
    }
}

// ---- finishing (src/cuda/tail.cu) ------------------------------------------------------

// Natural endpoint, peak repair and scale, one warp per job (tail.cu:83-139).
__global__ void selectNativeKernel(BatchView b, FinishView f)
{
    const int jobIndex = int(blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5));
    const int lane = int(threadIdx.x & 31);
    if (jobIndex >= b.jobCount)
        return;
    const JobInfo job = b.jobs[jobIndex];
    const int blocks = (job.frames + kBlockFrames - 1) / kBlockFrames;
    float peak = 0;
    int end = 0;
    bool nonfinite = false;
    for (int base = 0; base < blocks; base += 32) {
        const int block = base + lane;
        bool bad = false, quiet = false;
        float blockPeak = 0;
        int blockEnd = 0;
        if (block < blocks) {
            const StereoStats stat = f.stereo[job.blockFirst + block];
            blockPeak = stat.peak;
            bad = !isfinite(stat.peak);
            const int first = block * kBlockFrames;
            blockEnd = min(job.limit, first + kBlockFrames);
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
        }
        const unsigned stop = __ballot_sync(0xffffffffu, bad || quiet);
        const int first = stop ? __ffs(stop) - 1 : 32;
        if (lane < first || (lane == first && quiet))
            peak = fmaxf(peak, blockPeak);
        if (stop) {
            const int endLane = first;
            nonfinite = __shfl_sync(0xffffffffu, bad ? 1 : 0, endLane) != 0;
            end = __shfl_sync(0xffffffffu, blockEnd, endLane);
            break;
        }
    }
    #pragma unroll
    for (int d = 16; d; d >>= 1)
        peak = fmaxf(peak, __shfl_xor_sync(0xffffffffu, peak, d));
    if (lane)
        return;
    cs_tail_result result{};
    if (nonfinite) {
        result.status = CS_TAIL_NONFINITE;
        f.results[jobIndex] = result;
        return;
    }
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

// Mono PCM16 with ties-to-even channel average and per-window stats (tail.cu:147-181).
__global__ void quantizeMonoKernel(BatchView b, FinishView f, int window)
{
    __shared__ double reduceD[32];
    __shared__ int reduceI[32];
    const int w = int(blockIdx.x);
    const int jobIndex = b.windowJob[w];
    const JobInfo job = b.jobs[jobIndex];
    const cs_tail_result& result = f.results[jobIndex];
    const int first = (w - job.windowFirst) * window;
    const int end = min(first + window, result.dataFrames);
    if (first >= end)
        return;
    const float scale = result.scale;
    const float2* mix = static_cast<const float2*>(b.mix) + job.offset;
    short* mono = f.mono + job.offset;
    double power = 0;
    int peak = 0;
    for (int frame = first + int(threadIdx.x); frame < end; frame += blockDim.x) {
        const float2 sample = mix[frame];
        const int left = __float2int_rn(fminf(32767.f, fmaxf(-32768.f, sample.x * scale)));
        const int right = __float2int_rn(fminf(32767.f, fmaxf(-32768.f, sample.y * scale)));
        const int sum = left + right;
        const int value = (sum >> 1) + ((sum & 1) & ((sum >> 1) & 1));
        mono[frame] = short(value);
        power += double(value) * value;
        peak = max(peak, abs(value));
    }
    power = blockReduce(power, 0.0, SumOp{}, reduceD);
    peak = blockReduce(peak, 0, MaxOp{}, reduceI);
    if (threadIdx.x == 0)
        f.windows[w] = {power, peak};
}

// Weak-tail trim, one warp per job (tail.cu:183-213).
__global__ void selectTrimKernel(BatchView b, FinishView f, TailConfig config)
{
    const int jobIndex = int(blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5));
    const int lane = int(threadIdx.x & 31);
    if (jobIndex >= b.jobCount)
        return;
    cs_tail_result& result = f.results[jobIndex];
    if (result.status != CS_TAIL_OK)
        return;
    const MonoStats* windows = f.windows + b.jobs[jobIndex].windowFirst;
    const int count = (result.dataFrames + config.window - 1) / config.window;
    double maxPower = 0;
    for (int i = lane; i < count; i += 32)
        maxPower = fmax(maxPower, windows[i].power);
    #pragma unroll
    for (int d = 16; d; d >>= 1)
        maxPower = fmax(maxPower, __shfl_xor_sync(0xffffffffu, maxPower, d));
    const double threshold = fmin(config.ceiling, fmax(config.floor, sqrt(maxPower / config.window) * config.relative));
    int last = -1;
    for (int top = count - 1; top >= 0 && last < 0; top -= 32) {
        const int i = top - lane;
        const bool loud = i >= 0 && (sqrt(windows[i].power / config.window) > threshold || windows[i].peak > threshold * 4);
        const unsigned hits = __ballot_sync(0xffffffffu, loud);
        if (hits)
            last = top - (__ffs(hits) - 1);
    }
    if (lane || last < 0)
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

__device__ __forceinline__ short fadeSample(short value, int index, int count)
{
    constexpr double pi = 3.14159265358979323846;
    const double gain = count == 1 ? 0 : .5 * (1 + cos(pi * index / (count - 1)));
    return short(__double2int_rn(value * gain));
}

// Fade, compaction and peak / audible range (tail.cu:240-297).
template <int Channels>
__global__ void finalizeKernel(BatchView b, FinishView f, const short* input, int quality)
{
    __shared__ int reduceI[32];
    const int block = int(blockIdx.x);
    const int jobIndex = b.blockJob[block];
    const JobInfo job = b.jobs[jobIndex];
    cs_tail_result& result = f.results[jobIndex];
    const uint64_t outputOffset = result.offset;
    const int frames = result.frames, fade = result.fade;
    const int first = (block - job.blockFirst) * kBlockFrames;
    const int end = min(first + kBlockFrames, result.dataFrames);
    if (first >= end)
        return;
    int peak = 0, audibleFirst = frames, audibleLast = -1, clipped = 0;
    const int fadeStart = frames - fade;
    for (int frame = first + int(threadIdx.x); frame < end; frame += blockDim.x) {
        int framePeak = 0;
        #pragma unroll
        for (int c = 0; c < Channels; ++c) {
            short value = input[(job.offset + frame) * Channels + c];
            if (frame >= fadeStart)
                value = fadeSample(value, frame - fadeStart, fade);
            f.packed[(outputOffset + frame) * Channels + c] = value;
            const int magnitude = abs(int(value));
            framePeak = max(framePeak, magnitude);
            clipped += magnitude >= 32767;
        }
        peak = max(peak, framePeak);
        if (framePeak > 3) {
            audibleFirst = min(audibleFirst, frame);
            audibleLast = frame;
        }
    }
    peak = blockReduce(peak, 0, MaxOp{}, reduceI);
    audibleFirst = blockReduce(audibleFirst, frames, MinOp{}, reduceI);
    audibleLast = blockReduce(audibleLast, -1, MaxOp{}, reduceI);
    clipped = blockReduce(clipped, 0, SumOp{}, reduceI);
    if (threadIdx.x == 0) {
        if (quality && clipped)
            atomicAdd(&result.audio.clipped, clipped);
        if (audibleLast >= 0) {
            atomicMax(&result.peak, peak);
            atomicMin(&result.first, audibleFirst);
            atomicMax(&result.last, audibleLast);
        }
    }
}

// ---- launchers --------------------------------------------------------------------------

void launchPitch(const BatchView& b, const SegmentView& s, cudaStream_t stream)
{
    if (!s.pitchCount)
        return;
    pitchKernel<<<(s.pitchCount + 63) / 64, 64, 0, stream>>>(b, s);
}

void launchChains(const BatchView& b, const SegmentView& s, cudaStream_t stream)
{
    if (!s.chainCount)
        return;
    chainKernel<<<(s.chainCount + kChainWarps - 1) / kChainWarps, kChainWarps * 32, 0, stream>>>(b, s);
}

void launchMix(const BatchView& b, const SegmentView& s, bool natural, StereoStats* stats, cudaStream_t stream)
{
    if (!s.blockCount)
        return;
    if (natural)
        mixKernel<true><<<s.blockCount, kMixThreads, 0, stream>>>(b, s, stats);
    else
        mixKernel<false><<<s.blockCount, kMixThreads, 0, stream>>>(b, s, stats);
}

int launchFinish(const BatchView& b, const FinishView& f, bool natural, bool quality, const TailConfig& tail,
                 cudaStream_t stream)
{
    int launches = 0;
    const int warpsGrid = (b.jobCount + 7) / 8;
    if (natural) {
        selectNativeKernel<<<warpsGrid, 256, 0, stream>>>(b, f);
        ++launches;
        if (f.windowCount) {
            quantizeMonoKernel<<<f.windowCount, 256, 0, stream>>>(b, f, tail.window);
            ++launches;
        }
        selectTrimKernel<<<warpsGrid, 256, 0, stream>>>(b, f, tail);
        ++launches;
    }
    layoutKernel<<<1, 32, 0, stream>>>(b, f, natural ? 1 : 0);
    ++launches;
    if (f.blockCount) {
        if (natural)
            finalizeKernel<1><<<f.blockCount, 128, 0, stream>>>(b, f, f.mono, quality ? 1 : 0);
        else
            finalizeKernel<2><<<f.blockCount, 128, 0, stream>>>(b, f, static_cast<const short*>(b.mix),
                                                              quality ? 1 : 0);
        ++launches;
    }
    return launches;
}

} // namespace cs
