/*
 * ORACLE (test infrastructure, never shipped or measured): plain-C restatement of
 * the reference's per-voice render math, src/cuda/render.cu, and of the batch
 * index its renderer builds (src/cuda/renderer.cpp:390-460), run unsegmented in
 * the reference's launch order (renderer.cpp:1095-1106): variable pitch ->
 * filter sources -> voice filters -> mix tiles.
 *
 * Every function cites the reference lines it follows and keeps their operation
 * order; compiled with -ffp-contract=off it reproduces the reference built for
 * the host (oracle/_ref) bit for bit, which tests/test_oracle.py checks.  Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/claysampler_b200.h"

#define TAPS 48                 /* render.cu:3 */
#define PHASES 2048             /* render.cu:4 */
#define TILE 256

typedef struct { float x, y; } F2;
typedef struct { float b0, b1, b2, a1, a2; } Coeff;

typedef struct {                /* VoiceState, render_types.h:22-28 */
    double position, step;
    int pitchSpan, previousLoopEnd, previousLoopStart;
    int pitchInitialized, filterInitialized;
    float z1[CS_FILTER_SLOTS][3][2], z2[CS_FILTER_SLOTS][3][2];
    Coeff coefficients[CS_FILTER_SLOTS];
} State;

typedef struct {                /* Tile, render_types.h:70-74 */
    uint64_t output;
    int frame, frames, first, count;
    int controls[4];
} Tile;

typedef struct {
    const float* bank;
    const float* sinc;          /* tap-major [48][2049], as the reference */
    const double* sinc64;       /* the same table before its FP32 rounding (FP64 resampler mode) */
    cs_voice_span* voices;
    int voiceCount;
    cs_control_point* points;
    cs_voice_modulation* modulation;
    Tile* tiles;
    int tileCount;
    int* indices;
    int* filterHeads;
    int filterHeadCount;
    int* pitchHeads;
    int pitchHeadCount;
    int (*filterTiles)[2];      /* span, frame */
    int filterTileCount;
    float* filtered;
    double* phase;
    State* states;
    int lastFrame;
} Batch;

static F2 f2(float x, float y) { F2 v = {x, y}; return v; }

/* renderer.cpp:347-376; `wide` receives the FP64 values before the FP32
 * rounding the reference applies (renderer.cpp:370-371), when not null. */
static void sincTableBoth(float* table, double* wide)
{
    const double beta = 8.5, pi = 3.14159265358979323846;
    double norm;
    {
        double sum = 1, term = 1;
        for (int i = 1; i < 30; ++i) {
            term *= beta * beta / (4 * i * i);
            sum += term;
            if (term < 1e-14) break;
        }
        norm = sum;
    }
    for (int tap = 0; tap < TAPS; ++tap) {
        for (int phase = 0; phase <= PHASES; ++phase) {
            const double x = tap - 23 - (double)phase / PHASES;
            const double f = x / 24;
            const double value = beta * sqrt(1 - f * f);
            double sum = 1, term = 1;
            for (int i = 1; i < 30; ++i) {
                term *= value * value / (4 * i * i);
                sum += term;
                if (term < 1e-14) break;
            }
            const double window = sum / norm;
            const double value64 = window * (x == 0 ? 1 : sin(pi * x) / (pi * x));
            if (table) table[tap * (PHASES + 1) + phase] = (float)value64;
            if (wide) wide[tap * (PHASES + 1) + phase] = value64;
        }
    }
}

static void sincTable(float* table) { sincTableBoth(table, NULL); }

/* render.cu:6-19 (amplitude, filter and pitch envelopes share the fields) */
static float envelopeSpan(const cs_voice_span* e, int frame)
{
    if (e->releaseStart >= 0 && frame >= e->releaseStart) {
        if (frame >= e->fadeStart) return fmaxf(0, e->fadeValue - (frame - e->fadeStart + 1) * e->fadeStep);
        return e->releaseValue * expf((frame - e->releaseStart + 1) * e->releaseRate);
    }
    if (frame < e->attackStart) return e->start;
    if (frame < e->holdStart) return fminf(1, e->start + (frame - e->attackStart + 1) * e->attackStep);
    if (frame < e->decayStart) return 1;
    if (e->decayRate == 0) return e->sustain;
    return fmaxf(e->sustain, expf((frame - e->decayStart + 1) * e->decayRate));
}

static float envelopeShape(const cs_envelope_shape* e, int frame)
{
    if (e->releaseStart >= 0 && frame >= e->releaseStart) {
        if (frame >= e->fadeStart) return fmaxf(0, e->fadeValue - (frame - e->fadeStart + 1) * e->fadeStep);
        return e->releaseValue * expf((frame - e->releaseStart + 1) * e->releaseRate);
    }
    if (frame < e->attackStart) return e->start;
    if (frame < e->holdStart) return fminf(1, e->start + (frame - e->attackStart + 1) * e->attackStep);
    if (frame < e->decayStart) return 1;
    if (e->decayRate == 0) return e->sustain;
    return fmaxf(e->sustain, expf((frame - e->decayStart + 1) * e->decayRate));
}

/* render.cu:21-28 */
static F2 fetch(const float* bank, const cs_voice_span* v, int frame)
{
    if (frame < 0 || frame >= v->sourceEnd) return f2(0, 0);
    const uint64_t index = v->sample + (uint64_t)frame * (uint64_t)v->channels;
    const float left = bank[index];
    return f2(left, v->channels == 1 ? left : bank[index + 1]);
}

/* render.cu:30-61 in FP64: the unrounded table, products and sums in double,
 * rounded to float once at the end.  Bounds the FP32 resampler's error
 * independently of the reference's own FP32 arithmetic. */
static F2 interpolateAt64(const float* bank, const double* sinc, const cs_voice_span* v, double pos)
{
    const int center = (int)floor(pos);
    if (pos == center) return fetch(bank, v, center);
    const int phase = (int)nearbyint((pos - center) * PHASES);
    double x = 0, y = 0;
    for (int tap = 0; tap < TAPS; ++tap) {
        const F2 s = fetch(bank, v, center - 23 + tap);
        const double w = sinc[tap * (PHASES + 1) + phase];
        x += w * (double)s.x;
        y += w * (double)s.y;
    }
    return f2((float)x, (float)y);
}

/* render.cu:30-61 */
static F2 interpolateAt(const float* bank, const float* sinc, const double* sinc64, const cs_voice_span* v,
                        double pos)
{
    if (sinc64) return interpolateAt64(bank, sinc64, v, pos);
    const int center = (int)floor(pos);
    if (pos == center) return fetch(bank, v, center);
    const int phase = (int)nearbyint((pos - center) * PHASES);
    F2 r = f2(0, 0);
    if (center >= 23 && center < v->sourceEnd - 24) {
        const uint64_t index = v->sample + (uint64_t)(center - 23) * (uint64_t)v->channels;
        if (v->channels == 1) {
            for (int tap = 0; tap < TAPS; ++tap)
                r.x = fmaf(sinc[tap * (PHASES + 1) + phase], bank[index + tap], r.x);
            r.y = r.x;
        } else {
            for (int tap = 0; tap < TAPS; ++tap) {
                const float w = sinc[tap * (PHASES + 1) + phase];
                r.x = fmaf(w, bank[index + 2 * tap], r.x);
                r.y = fmaf(w, bank[index + 2 * tap + 1], r.y);
            }
        }
    } else {
        for (int tap = 0; tap < TAPS; ++tap) {
            const F2 s = fetch(bank, v, center - 23 + tap);
            const float w = sinc[tap * (PHASES + 1) + phase];
            r.x = fmaf(w, s.x, r.x);
            r.y = fmaf(w, s.y, r.y);
        }
    }
    return r;
}

/* render.cu:63-100 */
static F2 interpolate(const float* bank, const float* sinc, const double* sinc64, const cs_voice_span* v, int frame,
                      double pos)
{
    if (pos < 0) {
        const int elapsed = frame - v->begin;
        double distance = elapsed;
        if (v->pitchSlope != 0) distance = expm1(v->pitchSlope * elapsed) / expm1(v->pitchSlope);
        pos = v->position + distance * v->step;
    }
    if (v->generator != CS_GEN_NONE) {
        if (v->generator == CS_GEN_NOISE) {
            unsigned bits = v->noiseSeed + (unsigned)(frame - v->noiseStart);
            bits = (bits ^ (bits >> 16)) * 0x7feb352du;
            bits = (bits ^ (bits >> 15)) * 0x846ca68bu;
            bits ^= bits >> 16;
            const float value = (float)(bits >> 8) * (2.f / 16777216.f) - 1;
            return f2(value, value);
        }
        const float value = v->generator == CS_GEN_SINE ? -sinf(6.28318530717958647692f * (float)(pos - floor(pos))) : 0.f;
        return f2(value, value);
    }
    const int period = v->loopEnd - v->loopFirst;
    if (v->loopEnd > 0 && pos >= v->loopEnd) pos = v->loopFirst + fmod(pos - v->loopFirst, (double)period);
    if (pos >= v->sourceEnd) return f2(0, 0);
    F2 sample = interpolateAt(bank, sinc, sinc64, v, pos);
    const int fadeStart = v->loopEnd - v->loopCrossfade;
    if (v->loopEnd > 0 && v->loopCrossfade > 0 && pos >= fadeStart) {
        const F2 entry = interpolateAt(bank, sinc, sinc64, v, pos - period);
        const float phase = (float)((pos - fadeStart) / v->loopCrossfade);
        const float blend = .5f - .5f * cosf(3.14159265358979323846f * phase);
        sample.x = fmaf(blend, entry.x - sample.x, sample.x);
        sample.y = fmaf(blend, entry.y - sample.y, sample.y);
    }
    return sample;
}

/* render.cu:102-105 */
static short pcm16(float value) { return (short)(int)nearbyintf(fminf(32767, fmaxf(-32768, value * 32768))); }

/* render.cu:107-126 */
static float controlAt(const cs_control_point* points, int low, int high, int frame)
{
    while (low + 1 < high) {
        const int mid = low + (high - low) / 2;
        if (points[mid].frame <= frame) low = mid;
        else high = mid;
    }
    return fmaf(points[low].step, frame - points[low].frame, points[low].value);
}

static float modulationAt(const cs_voice_modulation* m, const cs_control_point* points, int frame)
{
    float value = m->first < 0 ? m->depth : m->depth * controlAt(points, m->first, m->last, frame);
    if (m->shapeFirst >= 0) value *= controlAt(points, m->shapeFirst, m->shapeLast, frame);
    return value;
}

static const float quarterPi = .7853981633974483f;

/* render.cu:130-136 */
static F2 panGains(const cs_voice_span* v, float offset)
{
    if (offset == 0) return f2(v->left, v->right);
    const float p = fminf(1, fmaxf(-1, v->pan + offset));
    return f2(v->gain * cosf((1 + p) * quarterPi), v->gain * cosf((1 - p) * quarterPi));
}

/* render.cu:138-187 */
static F2 voiceAudio(const Batch* b, const cs_voice_span* v, float pan, int frame, int filterInput, double phase)
{
    float level = envelopeSpan(v, frame);
    if (level <= 0) return f2(0, 0);
    float db = 0, widthOffset = 0, positionOffset = 0;
    for (int j = v->firstModulation; j < v->firstModulation + v->modulationCount; ++j) {
        const cs_voice_modulation* m = &b->modulation[j];
        if (m->target > CS_MOD_POSITION) continue;
        const float value = modulationAt(m, b->points, frame);
        switch (m->target) {
        case CS_MOD_AMPLITUDE: level *= value; break;
        case CS_MOD_VOLUME: db += value; break;
        case CS_MOD_PAN: pan += value; break;
        case CS_MOD_WIDTH: widthOffset += value; break;
        case CS_MOD_POSITION: positionOffset += value; break;
        default: break;
        }
    }
    if (db != 0) level *= exp2f(db * .166096404744368f);
    const F2 sample = interpolate(b->bank, b->sinc, b->sinc64, v, frame, phase);
    if (filterInput && v->channels == 1) return f2(sample.x * level, sample.x * level);
    const F2 gains = panGains(v, pan);
    const float l = sample.x * gains.x, r = sample.y * gains.y;
    if (v->stereoMatrix) {
        float direct = v->widthDirect, cross = v->widthCross;
        if (widthOffset != 0) {
            const float width = fminf(1, fmaxf(-1, v->width + widthOffset));
            direct = cosf((1 - width) * quarterPi);
            cross = cosf((1 + width) * quarterPi);
        }
        float positionLeft = v->positionLeft, positionRight = v->positionRight;
        if (positionOffset != 0) {
            const float position = fminf(1, fmaxf(-1, v->stereoPosition + positionOffset));
            positionLeft = cosf((1 + position) * quarterPi);
            positionRight = cosf((1 - position) * quarterPi);
        }
        return f2(fmaf(r, cross, l * direct) * (level * positionLeft), fmaf(l, cross, r * direct) * (level * positionRight));
    }
    return f2(l * level, r * level);
}

/* render.cu:189-193 */
static float jobGain(const cs_control_point* points, const int* offsets, int frame)
{
    return controlAt(points, offsets[0], offsets[1], frame) * controlAt(points, offsets[1], offsets[2], frame);
}

/* render.cu:195-213 (one frame of a filter tile) */
static void filterSource(const Batch* b, int span, int frame)
{
    const cs_voice_span* v = &b->voices[span];
    if (frame >= v->end || frame < 0 || frame >= b->lastFrame) return;
    const int* offsets = v->filterControls;
    const double position = v->variablePitch ? b->phase[v->phaseOffset + (frame - v->begin)] : -1;
    const F2 sample = voiceAudio(b, v, controlAt(b->points, offsets[2], offsets[3], frame), frame, 1, position);
    const float gain = jobGain(b->points, offsets, frame);
    float* dst = b->filtered + v->filteredOffset + (uint64_t)(frame - v->begin) * v->channels;
    dst[0] = sample.x * gain;
    if (v->channels == 2) dst[1] = sample.y * gain;
}

/* render.cu:222-266 (unsegmented) */
static void preparePitch(const Batch* b, int head)
{
    const cs_voice_span* voices = b->voices;
    if (!voices[head].variablePitch) return;
    State* state = &b->states[head];
    double position = state->pitchInitialized ? state->position : voices[head].position;
    int previousLoopEnd = state->previousLoopEnd, previousLoopStart = state->previousLoopStart;
    for (int span = head; span >= 0; span = voices[span].nextFilteredSpan) {
        const cs_voice_span* v = &voices[span];
        const int resumed = state->pitchInitialized && state->pitchSpan == span;
        if (!resumed && !v->loopEnd && previousLoopEnd > 0 && position >= previousLoopEnd)
            position = previousLoopStart + fmod(position - previousLoopStart, (double)(previousLoopEnd - previousLoopStart));
        previousLoopEnd = v->loopEnd;
        previousLoopStart = v->loopFirst;
        const double slope = exp(v->pitchSlope);
        double step = resumed ? state->step : v->step;
        for (int frame = v->begin; frame < v->end; ++frame) {
            b->phase[v->phaseOffset + (frame - v->begin)] = position;
            float cents = 0;
            float depth = v->extraEnvelope[1].depth;
            for (int j = v->firstModulation; j < v->firstModulation + v->modulationCount; ++j) {
                const cs_voice_modulation* m = &b->modulation[j];
                if (m->target == CS_MOD_PITCH) cents += modulationAt(m, b->points, frame);
                if (m->target == CS_MOD_PITCHEG_DEPTH) depth += modulationAt(m, b->points, frame);
            }
            if (v->activeEnvelope[1]) cents += depth * envelopeShape(&v->extraEnvelope[1], frame);
            position += step * exp2f(fminf(24000, fmaxf(-24000, cents)) / 1200);
            step *= slope;
        }
        state->pitchInitialized = 1;
        state->pitchSpan = span;
        state->position = position;
        state->step = step;
        state->previousLoopEnd = previousLoopEnd;
        state->previousLoopStart = previousLoopStart;
    }
}

/* render.cu:278-310 */
static Coeff coefficients(int type, float cutoff, float resonance, int rate, float bandwidth, float gain)
{
    const float w = 6.28318530717958647692f * fminf(fminf(20000.f, rate * .499f), fmaxf(1.f, cutoff)) / rate;
    if (type == CS_FILTER_LOW1 || type == CS_FILTER_HIGH1) {
        const float p = expf(-w);
        if (type == CS_FILTER_LOW1) { Coeff c = {1 - p, 0, 0, -p, 0}; return c; }
        const float high = (1 + p) * .5f;
        Coeff c = {high, -high, 0, -p, 0};
        return c;
    }
    float s, c;
    sincosf(w, &s, &c);
    if (type == CS_FILTER_PEAK) {
        const float a = exp2f(fminf(60, fmaxf(-96, gain)) * .083048202372184f);
        const float width = fminf(12, fmaxf(.01f, bandwidth));
        const float alpha = s * sinhf(fminf(20, .346573590279973f * width * w / s));
        const float inv = 1 / (1 + alpha / a);
        const float mid = -2 * c * inv;
        Coeff r = {(1 + alpha * a) * inv, mid, (1 - alpha * a) * inv, mid, (1 - alpha / a) * inv};
        return r;
    }
    const float alpha = .5f * s * exp2f(-.166096404744368f * fminf(60, fmaxf(-60, resonance)));
    const float inv = 1.f / (1 + alpha);
    const float a1 = -2 * c * inv;
    const float a2 = (1 - alpha) * inv;
    if (type == CS_FILTER_BAND2 || type == CS_FILTER_BAND4 || type == CS_FILTER_BAND6) {
        Coeff r = {alpha * inv, 0, -alpha * inv, a1, a2};
        return r;
    }
    if (type == CS_FILTER_NOTCH2) { Coeff r = {inv, a1, inv, a1, a2}; return r; }
    const int high = type == CS_FILTER_HIGH2 || type == CS_FILTER_HIGH4 || type == CS_FILTER_HIGH6;
    const float bb = (1 + (high ? c : -c)) * .5f * inv;
    Coeff r = {bb, (high ? -2 : 2) * bb, bb, a1, a2};
    return r;
}

/* render.cu:312-319 */
static int sections(int type)
{
    if (type == CS_FILTER_NONE) return 0;
    if (type == CS_FILTER_PEAK) return 1;
    if (type >= CS_FILTER_LOW6) return 3;
    if (type >= CS_FILTER_LOW4) return 2;
    return 1;
}

/* render.cu:321-336 */
static void smooth(Coeff* current, const Coeff* target, float amount)
{
    current->b0 = fmaf(amount, target->b0 - current->b0, current->b0);
    current->b1 = fmaf(amount, target->b1 - current->b1, current->b1);
    current->b2 = fmaf(amount, target->b2 - current->b2, current->b2);
    current->a1 = fmaf(amount, target->a1 - current->a1, current->a1);
    current->a2 = fmaf(amount, target->a2 - current->a2, current->a2);
}

static float filterSample(float x, const Coeff* c, float* z1, float* z2)
{
    const float y = fmaf(c->b0, x, *z1);
    *z1 = fmaf(-c->a1, y, fmaf(c->b1, x, *z2));
    *z2 = fmaf(-c->a2, y, c->b2 * x);
    return y;
}

/* render.cu:338-448 (unsegmented) */
static void applyFilter(const Batch* b, int head)
{
    const cs_voice_span* voices = b->voices;
    int has = 0;
    for (int f = 0; f < CS_FILTER_SLOTS; ++f) has |= voices[head].filters[f].type != CS_FILTER_NONE;
    if (!has) return;
    State* state = &b->states[head];
    float z1[CS_FILTER_SLOTS][3][2], z2[CS_FILTER_SLOTS][3][2];
    Coeff current[CS_FILTER_SLOTS];
    memcpy(z1, state->z1, sizeof z1);
    memcpy(z2, state->z2, sizeof z2);
    memcpy(current, state->coefficients, sizeof current);
    int initialized = state->filterInitialized;
    for (int span = head; span >= 0; span = voices[span].nextFilteredSpan) {
        const cs_voice_span* v = &voices[span];
        const int rate = v->sampleRate;
        const float amount = 1 - expf(-1000.f / rate);
        int count[CS_FILTER_SLOTS];
        int sectionCount = 0, firstSlot = 0;
        for (int f = 0; f < CS_FILTER_SLOTS; ++f) {
            count[f] = sections(v->filters[f].type);
            if (count[f]) firstSlot = f;
            sectionCount += count[f];
        }
        int moving = v->activeEnvelope[0] != 0;
        for (int j = v->firstModulation; j < v->firstModulation + v->modulationCount; ++j) {
            const int target = b->modulation[j].target;
            moving |= (target >= CS_MOD_CUTOFF && target <= CS_MOD_RESONANCE2) || target == CS_MOD_FILEG_DEPTH ||
                target >= CS_MOD_EQ1_FREQUENCY;
        }
        for (int frame = v->begin; frame < v->end; ++frame) {
            if (moving || !initialized) {
                float cents[2] = {0, 0}, db[2] = {0, 0}, eq[3][3] = {{0}};
                float depth = v->extraEnvelope[0].depth;
                for (int j = v->firstModulation; j < v->firstModulation + v->modulationCount; ++j) {
                    const cs_voice_modulation* m = &b->modulation[j];
                    if (m->target == CS_MOD_CUTOFF) cents[0] += modulationAt(m, b->points, frame);
                    if (m->target == CS_MOD_CUTOFF2) cents[1] += modulationAt(m, b->points, frame);
                    if (m->target == CS_MOD_RESONANCE) db[0] += modulationAt(m, b->points, frame);
                    if (m->target == CS_MOD_RESONANCE2) db[1] += modulationAt(m, b->points, frame);
                    if (m->target == CS_MOD_FILEG_DEPTH) depth += modulationAt(m, b->points, frame);
                    if (m->target >= CS_MOD_EQ1_FREQUENCY) {
                        const int id = m->target - CS_MOD_EQ1_FREQUENCY;
                        eq[id / 3][id % 3] += modulationAt(m, b->points, frame);
                    }
                }
                if (v->activeEnvelope[0]) cents[0] += depth * envelopeShape(&v->extraEnvelope[0], frame);
                for (int f = 0; f < CS_FILTER_SLOTS; ++f) {
                    if (!count[f]) continue;
                    const cs_voice_filter* filter = &v->filters[f];
                    const Coeff target = f < 2
                        ? coefficients(filter->type, filter->cutoff * exp2f(cents[f] / 1200), filter->resonance + db[f], rate, 0, 0)
                        : coefficients(filter->type, filter->cutoff + eq[f - 2][0], 0, rate, filter->bandwidth + eq[f - 2][1],
                                       filter->gain + eq[f - 2][2]);
                    if (initialized) smooth(&current[f], &target, amount);
                    else current[f] = target;
                }
                initialized = 1;
            }
            float* sample = b->filtered + v->filteredOffset + (uint64_t)(frame - v->begin) * v->channels;
            if (!moving && sectionCount == 1) {
                const Coeff coeff = current[firstSlot];
                float* z1l = &z1[firstSlot][0][0], *z1r = &z1[firstSlot][0][1];
                float* z2l = &z2[firstSlot][0][0], *z2r = &z2[firstSlot][0][1];
                for (int i = frame; i < v->end; ++i, sample += v->channels) {
                    sample[0] = filterSample(sample[0], &coeff, z1l, z2l);
                    if (v->channels == 2) sample[1] = filterSample(sample[1], &coeff, z1r, z2r);
                }
                break;
            }
            float left = sample[0];
            float right = v->channels == 2 ? sample[1] : 0.f;
            for (int f = 0; f < CS_FILTER_SLOTS; ++f) {
                for (int s = 0; s < count[f]; ++s) {
                    left = filterSample(left, &current[f], &z1[f][s][0], &z2[f][s][0]);
                    if (v->channels == 2) right = filterSample(right, &current[f], &z1[f][s][1], &z2[f][s][1]);
                }
            }
            sample[0] = left;
            if (v->channels == 2) sample[1] = right;
        }
    }
    state->filterInitialized = initialized;
    memcpy(state->z1, z1, sizeof z1);
    memcpy(state->z2, z2, sizeof z2);
    memcpy(state->coefficients, current, sizeof current);
}

/* render.cu:458-492 */
static F2 mixFrame(const Batch* b, const Tile* tile, int frame)
{
    const float pan = controlAt(b->points, tile->controls[2], tile->controls[3], frame);
    float left = 0, right = 0, wetLeft = 0, wetRight = 0;
    for (int i = tile->first; i < tile->first + tile->count; ++i) {
        const cs_voice_span* v = &b->voices[b->indices[i]];
        if (frame < v->begin || frame >= v->end) continue;
        if (v->filterTrack >= 0) {
            const float* source = b->filtered + v->filteredOffset + (uint64_t)(frame - v->begin) * v->channels;
            F2 sample = f2(source[0], v->channels == 1 ? source[0] : source[1]);
            if (v->channels == 1) {
                float offset = pan;
                for (int j = v->firstModulation; j < v->firstModulation + v->modulationCount; ++j)
                    if (b->modulation[j].target == CS_MOD_PAN) offset += modulationAt(&b->modulation[j], b->points, frame);
                const F2 gains = panGains(v, offset);
                sample.x *= gains.x;
                sample.y *= gains.y;
            }
            wetLeft += sample.x;
            wetRight += sample.y;
        } else {
            const F2 sample = voiceAudio(b, v, pan, frame, 0, -1);
            left += sample.x;
            right += sample.y;
        }
    }
    const float amplitude = jobGain(b->points, tile->controls, frame);
    return f2(fmaf(left, amplitude, wetLeft), fmaf(right, amplitude, wetRight));
}

/* BatchIndex::append (renderer.cpp:390-460) for a list of plans. */
static int buildBatch(Batch* b, const cs_plan* plans, int count)
{
    int spans = 0, tiles = 0, points = 0, mods = 0, indices = 0, chains = 0, filterTiles = 0;
    size_t filtered = 0, pitch = 0;
    for (int j = 0; j < count; ++j) {
        const cs_plan* p = &plans[j];
        spans += p->span_count;
        tiles += (p->frames + TILE - 1) / TILE;
        points += (int)(p->track_offsets[p->track_count] - p->track_offsets[0]);
        mods += p->modulation_count;
        for (int s = 0; s < p->span_count; ++s) {
            const cs_voice_span* v = &p->spans[s];
            indices += (v->end - 1) / TILE - v->begin / TILE + 1;
            if (v->filterTrack >= 0) {
                filtered += (size_t)(v->end - v->begin) * v->channels;
                if (v->variablePitch) pitch += (size_t)(v->end - v->begin);
                filterTiles += (v->end - v->begin + TILE - 1) / TILE;
                ++chains;
            }
        }
        if (b->lastFrame < p->frames) b->lastFrame = p->frames;
    }
    b->voices = calloc((size_t)spans + 1, sizeof *b->voices);
    b->tiles = calloc((size_t)tiles + 1, sizeof *b->tiles);
    b->points = calloc((size_t)points + 1, sizeof *b->points);
    b->modulation = calloc((size_t)mods + 1, sizeof *b->modulation);
    b->indices = calloc((size_t)indices + 1, sizeof *b->indices);
    b->filterHeads = calloc((size_t)chains + 1, sizeof(int));
    b->pitchHeads = calloc((size_t)chains + 1, sizeof(int));
    b->filterTiles = calloc((size_t)filterTiles + 1, sizeof *b->filterTiles);
    b->filtered = calloc(filtered + 1, sizeof(float));
    b->phase = calloc(pitch + 1, sizeof(double));
    b->states = calloc((size_t)spans + 1, sizeof *b->states);
    if (!b->voices || !b->tiles || !b->points || !b->modulation || !b->indices || !b->filterHeads || !b->pitchHeads ||
        !b->filterTiles || !b->filtered || !b->phase || !b->states)
        return -1;
    uint64_t frames = 0;
    size_t filteredOffset = 0, pitchOffset = 0;
    int voiceCount = 0, tileCount = 0, pointCount = 0, modCount = 0, indexCount = 0;
    for (int j = 0; j < count; ++j) {
        const cs_plan* p = &plans[j];
        const int tileN = (p->frames + TILE - 1) / TILE;
        int* offsets = calloc((size_t)tileN + 1, sizeof(int));
        int* controlOffsets = calloc((size_t)p->track_count + 1, sizeof(int));
        int* tails = malloc(sizeof(int) * (size_t)(p->filter_tracks + 1));
        for (int t = 0; t < p->filter_tracks; ++t) tails[t] = -1;
        for (int s = 0; s < p->span_count; ++s) {
            ++offsets[p->spans[s].begin / TILE];
            --offsets[(p->spans[s].end - 1) / TILE + 1];
        }
        for (int t = 1; t <= tileN; ++t) offsets[t] += offsets[t - 1];
        controlOffsets[0] = pointCount;
        for (int i = 0; i < p->track_count; ++i) {
            const int64_t n = p->track_offsets[i + 1] - p->track_offsets[i];
            memcpy(b->points + pointCount, p->points + p->track_offsets[i], (size_t)n * sizeof(cs_control_point));
            pointCount += (int)n;
            controlOffsets[i + 1] = pointCount;
        }
        const int modulationOffset = modCount;
        for (int m = 0; m < p->modulation_count; ++m) {
            cs_voice_modulation binding = p->modulation[m];
            if (binding.first >= 0) {
                binding.last = controlOffsets[binding.first + 1];
                binding.first = controlOffsets[binding.first];
            }
            if (binding.shapeFirst >= 0) {
                binding.shapeLast = controlOffsets[binding.shapeFirst + 1];
                binding.shapeFirst = controlOffsets[binding.shapeFirst];
            }
            b->modulation[modCount++] = binding;
        }
        for (int t = 0; t < tileN; ++t) {
            const int frame = t * TILE;
            Tile tile = {frames + (uint64_t)frame, frame, p->frames - frame < TILE ? p->frames - frame : TILE,
                         indexCount, offsets[t], {0, 0, 0, 0}};
            memcpy(tile.controls, controlOffsets, 4 * sizeof(int));
            b->tiles[tileCount++] = tile;
            indexCount += offsets[t];
            offsets[t] = tile.first;
        }
        for (int s = 0; s < p->span_count; ++s) {
            cs_voice_span voice = p->spans[s];
            const int index = voiceCount;
            for (int t = voice.begin / TILE; t <= (voice.end - 1) / TILE; ++t) b->indices[offsets[t]++] = index;
            voice.firstModulation += modulationOffset;
            if (voice.filterTrack >= 0) {
                int* tail = &tails[voice.filterTrack];
                if (*tail < 0) {
                    if (voice.variablePitch) b->pitchHeads[b->pitchHeadCount++] = index;
                    int any = 0;
                    for (int f = 0; f < CS_FILTER_SLOTS; ++f) any |= voice.filters[f].type != CS_FILTER_NONE;
                    if (any) b->filterHeads[b->filterHeadCount++] = index;
                } else {
                    b->voices[*tail].nextFilteredSpan = index;
                }
                *tail = index;
                voice.nextFilteredSpan = -1;
                voice.filteredOffset = filteredOffset;
                filteredOffset += (size_t)(voice.end - voice.begin) * voice.channels;
                if (voice.variablePitch) {
                    voice.phaseOffset = pitchOffset;
                    pitchOffset += (size_t)(voice.end - voice.begin);
                }
                memcpy(voice.filterControls, controlOffsets, 4 * sizeof(int));
                for (int frame = voice.begin; frame < voice.end; frame += TILE) {
                    b->filterTiles[b->filterTileCount][0] = index;
                    b->filterTiles[b->filterTileCount][1] = frame;
                    ++b->filterTileCount;
                }
            }
            b->voices[voiceCount++] = voice;
        }
        frames += (uint64_t)p->frames;
        free(offsets);
        free(controlOffsets);
        free(tails);
    }
    b->voiceCount = voiceCount;
    b->tileCount = tileCount;
    return 0;
}

static void freeBatch(Batch* b)
{
    free(b->voices); free(b->tiles); free(b->points); free(b->modulation); free(b->indices);
    free(b->filterHeads); free(b->pitchHeads); free(b->filterTiles); free(b->filtered); free(b->phase);
    free(b->states);
}

static int synthesize(const cs_plan* plans, int count, const float* bank, int natural, int threads, void* out,
                      int fp64)
{
    static float* sinc = NULL;
    static double* sinc64 = NULL;
    #pragma omp critical(oracle_sinc)
    {
        if (!sinc) {
            float* table = malloc(sizeof(float) * TAPS * (PHASES + 1));
            double* wide = malloc(sizeof(double) * TAPS * (PHASES + 1));
            sincTableBoth(table, wide);
            sinc64 = wide;
            sinc = table;
        }
    }
    Batch b;
    memset(&b, 0, sizeof b);
    b.bank = bank;
    b.sinc = sinc;
    b.sinc64 = fp64 ? sinc64 : NULL;
    if (buildBatch(&b, plans, count)) {
        freeBatch(&b);
        return 1;
    }
    #pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
    for (int i = 0; i < b.pitchHeadCount; ++i) preparePitch(&b, b.pitchHeads[i]);
    #pragma omp parallel for schedule(dynamic, 16) num_threads(threads)
    for (int t = 0; t < b.filterTileCount; ++t)
        for (int lane = 0; lane < TILE; ++lane) filterSource(&b, b.filterTiles[t][0], b.filterTiles[t][1] + lane);
    #pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
    for (int i = 0; i < b.filterHeadCount; ++i) applyFilter(&b, b.filterHeads[i]);
    #pragma omp parallel for schedule(dynamic, 16) num_threads(threads)
    for (int t = 0; t < b.tileCount; ++t) {
        const Tile* tile = &b.tiles[t];
        for (int lane = 0; lane < tile->frames; ++lane) {
            const F2 mixed = mixFrame(&b, tile, tile->frame + lane);
            if (natural) {
                float* dst = (float*)out + 2 * (tile->output + (uint64_t)lane);
                dst[0] = mixed.x;
                dst[1] = mixed.y;
            } else {
                short* dst = (short*)out + 2 * (tile->output + (uint64_t)lane);
                dst[0] = pcm16(mixed.x);
                dst[1] = pcm16(mixed.y);
            }
        }
    }
    freeBatch(&b);
    return 0;
}

/* The batch's mix: float2 per frame (natural) or short2 (orig/custom), jobs
 * concatenated in plan order. */
int oracle_synthesize(const cs_plan* plans, int count, const float* bank, int natural, int threads, void* out)
{
    return synthesize(plans, count, bank, natural, threads, out, 0);
}

/* As oracle_synthesize with the resampler in FP64 (interpolateAt64); the rest of
 * the voice math stays the reference's FP32. */
int oracle_synthesize_fp64_resampler(const cs_plan* plans, int count, const float* bank, int natural, int threads,
                                     void* out)
{
    return synthesize(plans, count, bank, natural, threads, out, 1);
}

void oracle_sinc_table(float* out)
{
    sincTable(out);
}
