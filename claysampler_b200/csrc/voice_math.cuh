// Per-voice, per-frame arithmetic of the render path.  Each function restates the
// reference's definition (src/cuda/render.cu) operation for operation, because the
// float bus is checked against the reference within 1e-5 of full scale and PCM16 to
// one LSB.  The build contracts multiply-adds as the reference's NVRTC build does
// (nvcc's default), and with the same expressions the compiler fuses the same
// pairs: the mix comes out bit-identical to the reference's own kernels on the GPU.
#pragma once

#include "kernels.cuh"
#include <stdint.h>

namespace cs {

constexpr float kQuarterPi = .7853981633974483f;

// Amplitude / filter / pitch envelope value at `frame` (render.cu:6-19).
template <class Shape>
__device__ __forceinline__ float envelopeAt(const Shape& e, int frame)
{
    if (e.releaseStart >= 0 && frame >= e.releaseStart) {
        if (frame >= e.fadeStart)
            return fmaxf(0.f, e.fadeValue - float(frame - e.fadeStart + 1) * e.fadeStep);
        return e.releaseValue * expf(float(frame - e.releaseStart + 1) * e.releaseRate);
    }
    if (frame < e.attackStart) return e.start;
    if (frame < e.holdStart) return fminf(1.f, e.start + float(frame - e.attackStart + 1) * e.attackStep);
    if (frame < e.decayStart) return 1.f;
    if (e.decayRate == 0) return e.sustain;
    return fmaxf(e.sustain, expf(float(frame - e.decayStart + 1) * e.decayRate));
}

#ifndef CS_TRACK_WINDOW
#define CS_TRACK_WINDOW 4
#endif

// Binary search for the last point with point.frame <= frame in [below, above),
// given points[below].frame <= frame < points[above].frame.
__device__ __forceinline__ int searchPoints(const cs_control_point* __restrict__ points, int below, int above, int frame)
{
    while (below + 1 < above) {
        const int mid = below + (above - below) / 2;
        if (__ldg(&points[mid].frame) <= frame) below = mid;
        else above = mid;
    }
    return below;
}

// Index of the last point with point.frame <= frame in [low, high) of a track whose
// frames do not decrease, or `low` when there is none: the point the reference's
// binary search lands on (render.cu:107-118).  Past the track's first point, a
// guess interpolated between its second and last points (right or off by one for
// evenly spaced points, such as an LFO baked every 16 frames after its start
// anchor) bounds a window of 2 x CS_TRACK_WINDOW points; when the window holds the
// answer the search takes a few steps inside it, otherwise it falls back to the
// whole track.  Either way the index is the one the binary search finds.
__device__ __forceinline__ int pointAt(const cs_control_point* __restrict__ points, int low, int high, int frame)
{
    if (high - low <= 1)
        return low;
    const int second = low + 1;
    const int secondFrame = __ldg(&points[second].frame), lastFrame = __ldg(&points[high - 1].frame);
    if (frame >= lastFrame)
        return high - 1;
    if (frame < secondFrame)
        return low;                     // whether or not the first point is due
    // secondFrame <= frame < lastFrame: the answer lies in [second, high - 2].
    const float scale = __fdividef(float(high - 1 - second), float(lastFrame - secondFrame));
    const int guess = second + __float2int_rz(float(frame - secondFrame) * scale);
    const int below = max(second, guess - CS_TRACK_WINDOW), above = min(high - 1, guess + CS_TRACK_WINDOW);
    if (below < above && __ldg(&points[below].frame) <= frame && __ldg(&points[above].frame) > frame)
        return searchPoints(points, below, above, frame);
    return searchPoints(points, second, high - 1, frame);
}

// Piecewise-linear track value at the point pointAt finds (render.cu:107-118).
__device__ __forceinline__ float trackAt(const cs_control_point* __restrict__ points, int low, int high, int frame)
{
    const int at = pointAt(points, low, high, frame);
    return fmaf(__ldg(&points[at].step), float(frame - __ldg(&points[at].frame)), __ldg(&points[at].value));
}

__device__ __forceinline__ float bindingAt(const cs_voice_modulation& m, const cs_control_point* __restrict__ points,
                                           int frame)
{
    float value = m.first < 0 ? m.depth : m.depth * trackAt(points, m.first, m.last, frame);
    if (m.shapeFirst >= 0)
        value *= trackAt(points, m.shapeFirst, m.shapeLast, frame);
    return value;
}

// CC7 x CC11 job gain (render.cu:189-193); `tracks` holds the job's first four
// track point offsets.
__device__ __forceinline__ float jobGainAt(const cs_control_point* __restrict__ points, const int* tracks, int frame)
{
    return trackAt(points, tracks[0], tracks[1], frame) * trackAt(points, tracks[1], tracks[2], frame);
}

// Source frame with zero outside [0, sourceEnd) (render.cu:21-28).
__device__ __forceinline__ float2 sourceFrame(const float* __restrict__ bank, const cs_voice_span& v, int frame)
{
    if (frame < 0 || frame >= v.sourceEnd)
        return make_float2(0.f, 0.f);
    const uint64_t index = v.sample + uint64_t(frame) * uint64_t(v.channels);
    const float left = __ldg(bank + index);
    return make_float2(left, v.channels == 1 ? left : __ldg(bank + index + 1));
}

// Eight consecutive weights of a sinc row: one 256-bit load (sm_100), so a warp's
// request brings each lane a whole 32-byte sector of its own row.  `p` is 32-byte
// aligned: rows are 192 bytes and the table starts on a 256-byte boundary.
struct Weights8 {
    float w[8];
};

__device__ __forceinline__ Weights8 sincWeights8(const float* p)
{
    Weights8 r;
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(r.w[0]), "=f"(r.w[1]), "=f"(r.w[2]), "=f"(r.w[3]), "=f"(r.w[4]), "=f"(r.w[5]), "=f"(r.w[6]),
          "=f"(r.w[7])
        : "l"(p));
    return r;
}

// Sinc weights from the phase-major table in global memory: taps 8q .. 8q + 7 of
// a phase's row in one 256-bit load.
struct GlobalSincRows {
    const float* __restrict__ sinc;
    __device__ __forceinline__ Weights8 operator()(int phase, int q) const
    {
        return sincWeights8(sinc + size_t(phase) * kTaps + 8 * q);
    }
};

// Sinc weights from a half table in shared memory: rows 0 .. kPhases / 2, one
// per phase, kSharedSincStride floats apart (16-byte aligned rows spread over the
// banks).  The table is symmetric, sinc[tap][phase] == sinc[47 - tap][2048 - phase]
// exactly (the two arguments are exact negatives, and the window and sin(x)/x are
// even), so a phase above 1024 reads row 2048 - phase backwards.
constexpr int kSharedSincStride = 52;
constexpr int kSharedSincRows = kPhases / 2 + 1;

struct SharedSincRows {
    const float* table;
    __device__ __forceinline__ Weights8 operator()(int phase, int q) const
    {
        Weights8 r;
        if (phase <= kPhases / 2) {
            const float4* row = reinterpret_cast<const float4*>(table + phase * kSharedSincStride + 8 * q);
            const float4 a = row[0], b = row[1];
            r.w[0] = a.x; r.w[1] = a.y; r.w[2] = a.z; r.w[3] = a.w;
            r.w[4] = b.x; r.w[5] = b.y; r.w[6] = b.z; r.w[7] = b.w;
        } else {
            // Taps 8q .. 8q + 7 are columns 47 - 8q down to 40 - 8q.
            const float* row = table + (kPhases - phase) * kSharedSincStride;
            const float4 a = *reinterpret_cast<const float4*>(row + 44 - 8 * q);
            const float4 b = *reinterpret_cast<const float4*>(row + 40 - 8 * q);
            r.w[0] = a.w; r.w[1] = a.z; r.w[2] = a.y; r.w[3] = a.x;
            r.w[4] = b.w; r.w[5] = b.z; r.w[6] = b.y; r.w[7] = b.x;
        }
        return r;
    }
};

// 48-tap windowed-sinc value at `pos` (render.cu:30-61), the weights of a phase
// eight at a time from `rows`; the tap order of the accumulation is unchanged.
template <bool VectorTaps, class Rows>
__device__ __forceinline__ float2 sincAtRows(const float* __restrict__ bank, const Rows& rows,
                                             const cs_voice_span& v, double pos)
{
    const int center = __double2int_rd(pos);
    if (pos == double(center))
        return sourceFrame(bank, v, center);
    const int phase = __double2int_rn((pos - double(center)) * kPhases);
    float x = 0.f, y = 0.f;
    if (center >= 23 && center < v.sourceEnd - 24) {
        const float* s = bank + v.sample + uint64_t(center - 23) * uint64_t(v.channels);
        const uint64_t first = v.sample + uint64_t(center - 23);     // float index of tap 0 (mono)
        const uint64_t base = first & ~uint64_t(3);
        if (VectorTaps && v.channels == 1 && base + 52 <= v.sample + uint64_t(v.sourceEnd)) {
            // The 48 taps from thirteen aligned 128-bit loads of the 52 floats around
            // them (all inside this sample), picked by the offset `first - base`
            // (VectorTaps: for kernels with the registers to hold them).
            const float4* s4 = reinterpret_cast<const float4*>(bank + base);
            const int offset = int(first - base);
            const bool odd = (offset & 1) != 0, two = (offset & 2) != 0;
            float4 lo = __ldg(s4);
            #pragma unroll
            for (int q = 0; q < kTaps / 8; ++q) {
                const Weights8 w = rows(phase, q);
                const float4 mid = __ldg(s4 + 2 * q + 1), hi = __ldg(s4 + 2 * q + 2);
                const float f[12] = {lo.x, lo.y, lo.z, lo.w, mid.x, mid.y, mid.z, mid.w, hi.x, hi.y, hi.z, hi.w};
                float g[10];
                #pragma unroll
                for (int i = 0; i < 10; ++i)
                    g[i] = odd ? f[i + 1] : f[i];
                #pragma unroll
                for (int k = 0; k < 8; ++k)
                    x = fmaf(w.w[k], two ? g[k + 2] : g[k], x);
                lo = hi;
            }
            y = x;
        } else if (v.channels == 1) {
            #pragma unroll
            for (int q = 0; q < kTaps / 8; ++q) {
                const Weights8 w = rows(phase, q);
                #pragma unroll
                for (int k = 0; k < 8; ++k)
                    x = fmaf(w.w[k], __ldg(s + 8 * q + k), x);
            }
            y = x;
        } else if ((reinterpret_cast<uintptr_t>(s) & 7) == 0) {
            const float2* s2 = reinterpret_cast<const float2*>(s);
            #pragma unroll
            for (int q = 0; q < kTaps / 8; ++q) {
                const Weights8 w = rows(phase, q);
                #pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const float2 pk = __ldg(s2 + 8 * q + k);
                    x = fmaf(w.w[k], pk.x, x);
                    y = fmaf(w.w[k], pk.y, y);
                }
            }
        } else {
            // A stereo sample that starts at an odd float offset (after an odd-length
            // mono sample in the bank) cannot use 8-byte loads.
            #pragma unroll 2
            for (int q = 0; q < kTaps / 8; ++q) {
                const Weights8 w = rows(phase, q);
                #pragma unroll
                for (int k = 0; k < 8; ++k) {
                    x = fmaf(w.w[k], __ldg(s + 2 * (8 * q + k)), x);
                    y = fmaf(w.w[k], __ldg(s + 2 * (8 * q + k) + 1), y);
                }
            }
        }
    } else {
        for (int q = 0; q < kTaps / 8; ++q) {
            const Weights8 w = rows(phase, q);
            #pragma unroll
            for (int k = 0; k < 8; ++k) {
                const float2 s = sourceFrame(bank, v, center - 23 + 8 * q + k);
                x = fmaf(w.w[k], s.x, x);
                y = fmaf(w.w[k], s.y, y);
            }
        }
    }
    return make_float2(x, y);
}

template <bool VectorTaps = false>
__device__ __forceinline__ float2 sincAt(const float* __restrict__ bank, const float* __restrict__ sinc,
                                         const cs_voice_span& v, double pos)
{
    return sincAtRows<VectorTaps>(bank, GlobalSincRows{sinc}, v, pos);
}

// fmod(x, period), which is exact.  For 0 <= x < 2^32 and a positive period it is
// the remainder of x's whole part (a 32-bit integer remainder) plus x's fraction:
// x - floor(x) is exact, and the sum is the exact remainder, so it is returned
// unrounded.  Other arguments go to fmod.
__device__ __forceinline__ double loopRemainder(double x, int period)
{
    if (x >= 0 && x < 4294967296.0 && period > 0) {
        const double whole = floor(x);
        return double(unsigned(whole) % unsigned(period)) + (x - whole);
    }
    return fmod(x, double(period));
}

// Source value of a voice at output `frame` (render.cu:63-100): position from the
// span's start (or a precomputed variable-pitch phase), generators, loop wrap and
// loop crossfade.
// A voice's source position `elapsed` frames into its span (render.cu:65-70).
__device__ __forceinline__ double sourcePosition(const cs_voice_span& v, int elapsed)
{
    double distance = elapsed;
    if (v.pitchSlope != 0)
        distance = expm1(v.pitchSlope * elapsed) / expm1(v.pitchSlope);
    return v.position + distance * v.step;
}

template <bool VectorTaps, class Rows>
__device__ __forceinline__ float2 voiceSourceRows(const float* __restrict__ bank, const Rows& rows,
                                                  const cs_voice_span& v, int frame, double pos)
{
    if (pos < 0)
        pos = sourcePosition(v, frame - v.begin);
    if (v.generator != CS_GEN_NONE) {
        if (v.generator == CS_GEN_NOISE) {
            unsigned bits = v.noiseSeed + unsigned(frame - v.noiseStart);
            bits = (bits ^ (bits >> 16)) * 0x7feb352du;
            bits = (bits ^ (bits >> 15)) * 0x846ca68bu;
            bits ^= bits >> 16;
            const float value = float(bits >> 8) * (2.f / 16777216.f) - 1.f;
            return make_float2(value, value);
        }
        const float value = v.generator == CS_GEN_SINE
            ? -sinf(6.28318530717958647692f * float(pos - floor(pos))) : 0.f;
        return make_float2(value, value);
    }
    const int period = v.loopEnd - v.loopFirst;
    if (v.loopEnd > 0 && pos >= v.loopEnd)
        pos = v.loopFirst + loopRemainder(pos - v.loopFirst, period);
    if (pos >= v.sourceEnd)
        return make_float2(0.f, 0.f);
    float2 sample = sincAtRows<VectorTaps>(bank, rows, v, pos);
    const int fadeStart = v.loopEnd - v.loopCrossfade;
    if (v.loopEnd > 0 && v.loopCrossfade > 0 && pos >= fadeStart) {
        const float2 entry = sincAtRows<VectorTaps>(bank, rows, v, pos - period);
        const float phase = float((pos - fadeStart) / v.loopCrossfade);
        const float blend = .5f - .5f * cosf(3.14159265358979323846f * phase);
        sample.x = fmaf(blend, entry.x - sample.x, sample.x);
        sample.y = fmaf(blend, entry.y - sample.y, sample.y);
    }
    return sample;
}

template <bool VectorTaps = false>
__device__ __forceinline__ float2 voiceSource(const float* __restrict__ bank, const float* __restrict__ sinc,
                                              const cs_voice_span& v, int frame, double pos)
{
    return voiceSourceRows<VectorTaps>(bank, GlobalSincRows{sinc}, v, frame, pos);
}

__device__ __forceinline__ short toPcm16(float value)
{
    return short(__float2int_rn(fminf(32767.f, fmaxf(-32768.f, value * 32768.f))));
}

// Constant-power pan gains (render.cu:130-136).
__device__ __forceinline__ float2 panGains(const cs_voice_span& v, float offset)
{
    if (offset == 0)
        return make_float2(v.left, v.right);
    const float p = fminf(1.f, fmaxf(-1.f, v.pan + offset));
    return make_float2(v.gain * cosf((1 + p) * kQuarterPi), v.gain * cosf((1 - p) * kQuarterPi));
}

// Modulation sums of one voice frame (render.cu:138-160): the enveloped level times
// the amplitude bindings, and the sums of the volume (dB), pan, width and
// position bindings, each accumulated in binding order.
struct VoiceMods {
    float level, db, pan, width, position;
};

__device__ __forceinline__ void addVoiceMod(VoiceMods& s, int target, float value)
{
    switch (target) {
    case CS_MOD_AMPLITUDE: s.level *= value; break;
    case CS_MOD_VOLUME: s.db += value; break;
    case CS_MOD_PAN: s.pan += value; break;
    case CS_MOD_WIDTH: s.width += value; break;
    case CS_MOD_POSITION: s.position += value; break;
    default: break;
    }
}

// The voice frame from its modulation sums and its source value `sample`
// (render.cu:160-187).  With `filterInput`, mono sources are returned before
// panning (the mix pans them after the filter).
__device__ __forceinline__ float2 voiceOutputFrom(float2 sample, const cs_voice_span& v, const VoiceMods& s,
                                                  bool filterInput)
{
    float level = s.level;
    if (s.db != 0)
        level *= exp2f(s.db * .166096404744368f);
    if (filterInput && v.channels == 1)
        return make_float2(sample.x * level, sample.x * level);
    const float2 gains = panGains(v, s.pan);
    const float l = sample.x * gains.x;
    const float r = sample.y * gains.y;
    if (v.stereoMatrix) {
        float direct = v.widthDirect, cross = v.widthCross;
        if (s.width != 0) {
            const float width = fminf(1.f, fmaxf(-1.f, v.width + s.width));
            direct = cosf((1 - width) * kQuarterPi);
            cross = cosf((1 + width) * kQuarterPi);
        }
        float positionLeft = v.positionLeft, positionRight = v.positionRight;
        if (s.position != 0) {
            const float position = fminf(1.f, fmaxf(-1.f, v.stereoPosition + s.position));
            positionLeft = cosf((1 + position) * kQuarterPi);
            positionRight = cosf((1 - position) * kQuarterPi);
        }
        return make_float2(fmaf(r, cross, l * direct) * (level * positionLeft),
                           fmaf(l, cross, r * direct) * (level * positionRight));
    }
    return make_float2(l * level, r * level);
}

// The voice frame from its modulation sums, resampling its source at `frame`.
template <bool VectorTaps = false>
__device__ __forceinline__ float2 voiceOutput(const float* __restrict__ bank, const float* __restrict__ sinc,
                                              const cs_voice_span& v, const VoiceMods& s, int frame,
                                              bool filterInput, double phase)
{
    return voiceOutputFrom(voiceSource<VectorTaps>(bank, sinc, v, frame, phase), v, s, filterInput);
}

// Modulation sums of one voice frame over its voice-level bindings, in binding
// order (render.cu:138-160); `level` is the enveloped level.
__device__ __forceinline__ VoiceMods voiceMods(const cs_voice_span& v, const cs_control_point* __restrict__ points,
                                               const cs_voice_modulation* __restrict__ modulation, float level,
                                               float pan, int frame)
{
    VoiceMods s{level, 0.f, pan, 0.f, 0.f};
    const int modEnd = v.firstModulation + v.modulationCount;
    for (int j = v.firstModulation; j < modEnd; ++j) {
        const cs_voice_modulation m = modulation[j];
        if (m.target > CS_MOD_POSITION)
            continue;
        addVoiceMod(s, m.target, bindingAt(m, points, frame));
    }
    return s;
}

// Enveloped, modulated, panned voice frame (render.cu:138-187).
template <bool VectorTaps = false>
__device__ __forceinline__ float2 voiceFrame(const float* __restrict__ bank, const float* __restrict__ sinc,
                                             const cs_voice_span& v, const cs_control_point* __restrict__ points,
                                             const cs_voice_modulation* __restrict__ modulation, float pan,
                                             int frame, bool filterInput, double phase)
{
    const float level = envelopeAt(v, frame);
    if (level <= 0)
        return make_float2(0.f, 0.f);
    const VoiceMods s = voiceMods(v, points, modulation, level, pan, frame);
    return voiceOutput<VectorTaps>(bank, sinc, v, s, frame, filterInput, phase);
}

// ---- filters (render.cu:276-336) ------------------------------------------------

struct Biquad {
    float b0, b1, b2, a1, a2;
};

__device__ __forceinline__ Biquad designFilter(int type, float cutoff, float resonance, int rate, float bandwidth,
                                               float gain)
{
    const float w = 6.28318530717958647692f * fminf(fminf(20000.f, float(rate) * .499f), fmaxf(1.f, cutoff)) /
        float(rate);
    if (type == CS_FILTER_LOW1 || type == CS_FILTER_HIGH1) {
        const float p = expf(-w);
        if (type == CS_FILTER_LOW1)
            return {1 - p, 0, 0, -p, 0};
        const float high = (1 + p) * .5f;
        return {high, -high, 0, -p, 0};
    }
    float s, c;
    sincosf(w, &s, &c);
    if (type == CS_FILTER_PEAK) {
        const float a = exp2f(fminf(60.f, fmaxf(-96.f, gain)) * .083048202372184f);
        const float width = fminf(12.f, fmaxf(.01f, bandwidth));
        const float alpha = s * sinhf(fminf(20.f, .346573590279973f * width * w / s));
        const float inv = 1 / (1 + alpha / a);
        const float mid = -2 * c * inv;
        return {(1 + alpha * a) * inv, mid, (1 - alpha * a) * inv, mid, (1 - alpha / a) * inv};
    }
    const float alpha = .5f * s * exp2f(-.166096404744368f * fminf(60.f, fmaxf(-60.f, resonance)));
    const float inv = 1.f / (1 + alpha);
    const float a1 = -2 * c * inv;
    const float a2 = (1 - alpha) * inv;
    if (type == CS_FILTER_BAND2 || type == CS_FILTER_BAND4 || type == CS_FILTER_BAND6)
        return {alpha * inv, 0, -alpha * inv, a1, a2};
    if (type == CS_FILTER_NOTCH2)
        return {inv, a1, inv, a1, a2};
    const bool high = type == CS_FILTER_HIGH2 || type == CS_FILTER_HIGH4 || type == CS_FILTER_HIGH6;
    const float b = (1 + (high ? c : -c)) * .5f * inv;
    return {b, (high ? -2 : 2) * b, b, a1, a2};
}

__device__ __forceinline__ int filterSections(int type)
{
    if (type == CS_FILTER_NONE) return 0;
    if (type == CS_FILTER_PEAK) return 1;
    if (type >= CS_FILTER_LOW6) return 3;
    if (type >= CS_FILTER_LOW4) return 2;
    return 1;
}

__device__ __forceinline__ void smoothToward(Biquad& current, const Biquad& target, float amount)
{
    current.b0 = fmaf(amount, target.b0 - current.b0, current.b0);
    current.b1 = fmaf(amount, target.b1 - current.b1, current.b1);
    current.b2 = fmaf(amount, target.b2 - current.b2, current.b2);
    current.a1 = fmaf(amount, target.a1 - current.a1, current.a1);
    current.a2 = fmaf(amount, target.a2 - current.a2, current.a2);
}

// Transposed direct form II step.
__device__ __forceinline__ float biquadStep(float x, const Biquad& c, float& z1, float& z2)
{
    const float y = fmaf(c.b0, x, z1);
    z1 = fmaf(-c.a1, y, fmaf(c.b1, x, z2));
    z2 = fmaf(-c.a2, y, c.b2 * x);
    return y;
}

// True when a span's filter coefficients change per frame (render.cu:370-375).
__device__ __forceinline__ bool filterMoves(const cs_voice_span& v, const cs_voice_modulation* __restrict__ modulation)
{
    bool moving = v.activeEnvelope[0] != 0;
    for (int j = v.firstModulation; j < v.firstModulation + v.modulationCount; ++j) {
        const int target = modulation[j].target;
        moving |= (target >= CS_MOD_CUTOFF && target <= CS_MOD_RESONANCE2) || target == CS_MOD_FILEG_DEPTH ||
            target >= CS_MOD_EQ1_FREQUENCY;
    }
    return moving;
}

// Target coefficients of every filter slot at `frame` (render.cu:378-405).
__device__ __forceinline__ void filterTargets(const cs_voice_span& v, const cs_control_point* __restrict__ points,
                                              const cs_voice_modulation* __restrict__ modulation, int frame,
                                              Biquad* out)
{
    float cents[2] = {0, 0}, db[2] = {0, 0};
    float eq[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    float depth = v.extraEnvelope[0].depth;
    for (int j = v.firstModulation; j < v.firstModulation + v.modulationCount; ++j) {
        const cs_voice_modulation m = modulation[j];
        if (m.target == CS_MOD_CUTOFF) cents[0] += bindingAt(m, points, frame);
        if (m.target == CS_MOD_CUTOFF2) cents[1] += bindingAt(m, points, frame);
        if (m.target == CS_MOD_RESONANCE) db[0] += bindingAt(m, points, frame);
        if (m.target == CS_MOD_RESONANCE2) db[1] += bindingAt(m, points, frame);
        if (m.target == CS_MOD_FILEG_DEPTH) depth += bindingAt(m, points, frame);
        if (m.target >= CS_MOD_EQ1_FREQUENCY) {
            const int id = m.target - CS_MOD_EQ1_FREQUENCY;
            eq[id / 3][id % 3] += bindingAt(m, points, frame);
        }
    }
    if (v.activeEnvelope[0])
        cents[0] += depth * envelopeAt(v.extraEnvelope[0], frame);
    for (int f = 0; f < CS_FILTER_SLOTS; ++f) {
        const cs_voice_filter& filter = v.filters[f];
        if (!filterSections(filter.type))
            continue;
        out[f] = f < 2 ? designFilter(filter.type, filter.cutoff * exp2f(cents[f] / 1200), filter.resonance + db[f],
                                      v.sampleRate, 0, 0)
                       : designFilter(filter.type, filter.cutoff + eq[f - 2][0], 0, v.sampleRate,
                                      filter.bandwidth + eq[f - 2][1], filter.gain + eq[f - 2][2]);
    }
}

} // namespace cs

namespace cs {

// Modulation sums of one of the two main filter slots (render.cu:378-396): cutoff
// cents, resonance dB and (slot 0) filter-envelope depth, in binding order.
struct FilterMods {
    float cents, db, depth;
};

__device__ __forceinline__ bool filterModTarget(int f, int target)
{
    return target == (f == 0 ? CS_MOD_CUTOFF : CS_MOD_CUTOFF2) ||
        target == (f == 0 ? CS_MOD_RESONANCE : CS_MOD_RESONANCE2) || (f == 0 && target == CS_MOD_FILEG_DEPTH);
}

__device__ __forceinline__ void addFilterMod(FilterMods& s, int f, int target, float value)
{
    if (target == (f == 0 ? CS_MOD_CUTOFF : CS_MOD_CUTOFF2)) s.cents += value;
    else if (target == (f == 0 ? CS_MOD_RESONANCE : CS_MOD_RESONANCE2)) s.db += value;
    else if (f == 0 && target == CS_MOD_FILEG_DEPTH) s.depth += value;
}

// Target coefficients of slot `f` from its modulation sums (render.cu:397-404).
__device__ __forceinline__ Biquad filterFromMods(const cs_voice_span& v, int f, const FilterMods& s, int frame)
{
    float cents = s.cents;
    if (f == 0 && v.activeEnvelope[0])
        cents += s.depth * envelopeAt(v.extraEnvelope[0], frame);
    const cs_voice_filter& filter = v.filters[f];
    return designFilter(filter.type, filter.cutoff * exp2f(cents / 1200), filter.resonance + s.db, v.sampleRate, 0, 0);
}

// The modulation sums of one frame of a filtered voice, for its output and for the
// target coefficients of its filter slot `f` (-1: none), in one pass over its
// bindings: each binding's value is computed once and added to the sum it feeds,
// and every sum keeps the reference's binding order (render.cu:138-160, 370-396).
// `moving` is filterMoves for the span.
struct SourceMods {
    VoiceMods voice;
    FilterMods filter;
    bool moving;
};

__device__ __forceinline__ SourceMods sourceMods(const cs_voice_span& v, const cs_control_point* __restrict__ points,
                                                 const cs_voice_modulation* __restrict__ modulation, float level,
                                                 float pan, int frame, int f)
{
    SourceMods s{{level, 0.f, pan, 0.f, 0.f}, {0.f, 0.f, v.extraEnvelope[0].depth}, v.activeEnvelope[0] != 0};
    const int end = v.firstModulation + v.modulationCount;
    for (int j = v.firstModulation; j < end; ++j) {
        const int target = modulation[j].target;
        s.moving |= (target >= CS_MOD_CUTOFF && target <= CS_MOD_RESONANCE2) || target == CS_MOD_FILEG_DEPTH ||
            target >= CS_MOD_EQ1_FREQUENCY;
        const bool voice = target <= CS_MOD_POSITION;
        const bool filter = f >= 0 && filterModTarget(f, target);
        if (!voice && !filter)
            continue;
        const float value = bindingAt(modulation[j], points, frame);
        if (voice)
            addVoiceMod(s.voice, target, value);
        else
            addFilterMod(s.filter, f, target, value);
    }
    return s;
}

// Target coefficients of one of the two main filter slots at `frame`; the same
// accumulation as filterTargets restricted to slot `f` (render.cu:378-404).
__device__ __forceinline__ Biquad filterTargetSlot(const cs_voice_span& v, const cs_control_point* __restrict__ points,
                                                   const cs_voice_modulation* __restrict__ modulation, int frame, int f)
{
    FilterMods s{0.f, 0.f, v.extraEnvelope[0].depth};
    for (int j = v.firstModulation; j < v.firstModulation + v.modulationCount; ++j) {
        const cs_voice_modulation m = modulation[j];
        if (filterModTarget(f, m.target))
            addFilterMod(s, f, m.target, bindingAt(m, points, frame));
    }
    return filterFromMods(v, f, s, frame);
}

} // namespace cs
