/*
 * ORACLE (test infrastructure, never shipped or measured): plain-C restatement of
 * the reference's GPU finishing stages, src/cuda/tail.cu, for the checker.
 *
 * Reductions follow the reference's launch shapes exactly: scanStereo sums each
 * 1024-frame block with 128 threads (thread t takes frames t, t+128, ...) followed
 * by the shuffle-down tree of tailReduce (tail.cu:13-30); the other reductions are
 * order-independent (max/min, or integer-valued sums that are exact in FP64).
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/claysampler_b200.h"

typedef struct { double power; float peak; } StereoStats;   /* render_types.h:142 */
typedef struct { double power; int peak; } MonoStats;       /* render_types.h:143 */

typedef struct {
    int window, quietFrames, padding, fade;
    double relative, floor, ceiling;
} OracleTailConfig;                                          /* render_types.h:100-103 */

/* tailReduce's two-level shuffle-down tree over `threads` per-thread sums. */
static double treeSum(const double* partial, int threads)
{
    double warps[32] = {0};
    const int count = threads / 32;
    for (int w = 0; w < count; ++w) {
        double v[32];
        memcpy(v, partial + 32 * w, sizeof v);
        for (int d = 16; d; d >>= 1)
            for (int lane = 0; lane < d; ++lane)
                v[lane] = v[lane] + v[lane + d];
        warps[w] = v[0];
    }
    double v[32];
    for (int lane = 0; lane < 32; ++lane)
        v[lane] = lane < count ? warps[lane] : 0.0;
    for (int d = 16; d; d >>= 1)
        for (int lane = 0; lane < d; ++lane)
            v[lane] = v[lane] + v[lane + d];
    return v[0];
}

/* scanStereo (tail.cu:54-75) for one block of one job. */
static StereoStats scanBlock(const float* mix, int first, int end)
{
    double partial[128];
    float peak = 0;
    for (int t = 0; t < 128; ++t) {
        double power = 0;
        for (int frame = first + t; frame < end; frame += 128) {
            const float x = mix[2 * frame], y = mix[2 * frame + 1];
            if (!isfinite(x) || !isfinite(y)) {
                peak = INFINITY;
                continue;
            }
            const float m = fmaxf(fabsf(x), fabsf(y));
            peak = fmaxf(peak, m);
            power += (double)(x * x) + (double)(y * y);
        }
        partial[t] = power;
    }
    StereoStats s = {treeSum(partial, 128), peak};
    return s;
}

/* selectNative (tail.cu:83-139). */
static cs_tail_result selectNative(const float* mix, const StereoStats* stats, const cs_plan* job)
{
    cs_tail_result result;
    memset(&result, 0, sizeof result);
    float peak = 0;
    int end = 0;
    for (int first = 0; first < job->frames; first += CS_TAIL_BLOCK_FRAMES) {
        const StereoStats stat = stats[first / CS_TAIL_BLOCK_FRAMES];
        if (!isfinite(stat.peak)) {
            result.status = CS_TAIL_NONFINITE;
            return result;
        }
        peak = fmaxf(peak, stat.peak);
        const int blockEnd = job->limit < first + CS_TAIL_BLOCK_FRAMES ? job->limit : first + CS_TAIL_BLOCK_FRAMES;
        if (blockEnd < job->music_end)
            continue;
        const double threshold = 1e-12 * (blockEnd - first) * 2;
        double power = stat.power;
        if (fabs(power - threshold) <= threshold * 1e-12) {
            power = 0;
            const int stop = blockEnd < job->frames ? blockEnd : job->frames;
            for (int frame = first; frame < stop; ++frame) {
                const float x = mix[2 * frame], y = mix[2 * frame + 1];
                power += x * x;
                power += y * y;
            }
        }
        if (power <= threshold) {
            end = blockEnd;
            break;
        }
    }
    if (!end) {
        const int silent = (job->frames + CS_TAIL_BLOCK_FRAMES - 1) / CS_TAIL_BLOCK_FRAMES * CS_TAIL_BLOCK_FRAMES;
        if (silent < job->limit) {
            const int music = (job->music_end + CS_TAIL_BLOCK_FRAMES - 1) / CS_TAIL_BLOCK_FRAMES * CS_TAIL_BLOCK_FRAMES;
            const int padded = silent + CS_TAIL_BLOCK_FRAMES > music ? silent + CS_TAIL_BLOCK_FRAMES : music;
            end = job->limit < padded ? job->limit : padded;
        }
    }
    if (!end) {
        result.status = CS_TAIL_DURATION;
    } else {
        const double attenuation = peak >= 1 ? 20 * log10((double)peak) + 1 : 0;
        if (attenuation > 5 + 1e-6) {
            result.status = CS_TAIL_PEAK;
        } else {
            result.frames = end;
            result.dataFrames = end < job->frames ? end : job->frames;
            result.scale = (float)(32768 * pow(10., -attenuation / 20));
        }
    }
    return result;
}

/* quantizeMono (tail.cu:147-174) for one job. */
static void quantizeMono(const float* mix, const cs_tail_result* result, int window, int16_t* mono, MonoStats* stats)
{
    const int windows = (result->dataFrames + window - 1) / window;
    for (int w = 0; w < windows; ++w) {
        const int first = w * window;
        const int end = first + window < result->dataFrames ? first + window : result->dataFrames;
        double power = 0;
        int peak = 0;
        for (int frame = first; frame < end; ++frame) {
            const int left = (int)nearbyintf(fminf(32767, fmaxf(-32768, mix[2 * frame] * result->scale)));
            const int right = (int)nearbyintf(fminf(32767, fmaxf(-32768, mix[2 * frame + 1] * result->scale)));
            const int sum = left + right;
            const int value = (sum >> 1) + ((sum & 1) & ((sum >> 1) & 1));
            mono[frame] = (int16_t)value;
            power += (double)value * value;
            peak = abs(value) > peak ? abs(value) : peak;
        }
        stats[w].power = power;
        stats[w].peak = peak;
    }
}

/* selectTrim (tail.cu:183-207). */
static void selectTrim(const MonoStats* windows, cs_tail_result* result, const OracleTailConfig* config)
{
    if (result->status != CS_TAIL_OK)
        return;
    const int count = (result->dataFrames + config->window - 1) / config->window;
    double maxPower = 0;
    for (int i = 0; i < count; ++i)
        maxPower = fmax(maxPower, windows[i].power);
    const double threshold = fmin(config->ceiling, fmax(config->floor, sqrt(maxPower / config->window) * config->relative));
    for (int i = count - 1; i >= 0; --i) {
        if (sqrt(windows[i].power / config->window) > threshold || windows[i].peak > threshold * 4) {
            const int sound = (i + 1) * config->window;
            const int lastSound = result->frames < sound ? result->frames : sound;
            if (result->frames - lastSound >= config->quietFrames) {
                result->frames = lastSound + config->padding;
                result->dataFrames = result->frames < result->dataFrames ? result->frames : result->dataFrames;
                result->fade = result->frames < config->fade ? result->frames : config->fade;
            }
            break;
        }
    }
}

static int16_t fadeSample(int16_t value, int index, int count)
{
    const double pi = 3.14159265358979323846;
    const double gain = count == 1 ? 0 : .5 * (1 + cos(pi * index / (count - 1)));
    return (int16_t)(int)nearbyint(value * gain);
}

/* finalizePcm (tail.cu:240-291) for one job.  Each 1024-frame block merges its
 * peak and audible range only when it holds an audible frame (tail.cu:286-290). */
static void finalize(const int16_t* input, int channels, cs_tail_result* result, int16_t* output, int quality)
{
    const int fadeStart = result->frames - result->fade;
    for (int first = 0; first < result->dataFrames; first += CS_TAIL_BLOCK_FRAMES) {
        const int end = first + CS_TAIL_BLOCK_FRAMES < result->dataFrames ? first + CS_TAIL_BLOCK_FRAMES
                                                                          : result->dataFrames;
        int peak = 0, audibleFirst = result->frames, audibleLast = -1;
        for (int frame = first; frame < end; ++frame) {
            int framePeak = 0;
            for (int c = 0; c < channels; ++c) {
                int16_t value = input[(size_t)frame * channels + c];
                if (frame >= fadeStart)
                    value = fadeSample(value, frame - fadeStart, result->fade);
                output[(size_t)frame * channels + c] = value;
                const int magnitude = abs((int)value);
                framePeak = magnitude > framePeak ? magnitude : framePeak;
                if (quality && magnitude >= 32767)
                    result->audio.clipped += 1;
            }
            peak = framePeak > peak ? framePeak : peak;
            if (framePeak > 3) {
                audibleFirst = frame < audibleFirst ? frame : audibleFirst;
                audibleLast = frame;
            }
        }
        if (audibleLast >= 0) {
            result->peak = peak > result->peak ? peak : result->peak;
            result->first = audibleFirst < result->first ? audibleFirst : result->first;
            result->last = audibleLast > result->last ? audibleLast : result->last;
        }
    }
}

/* Natural finishing of a batch: `mix` is float2 per frame with jobs concatenated.
 * Writes `count` results and the packed mono PCM16 (sum of dataFrames samples);
 * returns the packed sample count. */
size_t oracle_finish_natural(const float* mix, const cs_plan* plans, int count, int rate, int window, int quality,
                             cs_tail_result* results, int16_t* packed)
{
    OracleTailConfig config = {window, 2 * rate, (int)nearbyint(rate / 4.), (int)nearbyint(rate / 10.),
                               pow(10., -1.5), 32768 * pow(10., -3.9), 32768 * pow(10., -3.)};
    size_t offset = 0, frameBase = 0;
    for (int j = 0; j < count; ++j) {
        const cs_plan* job = &plans[j];
        const float* jobMix = mix + 2 * frameBase;
        const int blocks = (job->frames + CS_TAIL_BLOCK_FRAMES - 1) / CS_TAIL_BLOCK_FRAMES;
        StereoStats* stats = malloc(sizeof(StereoStats) * (size_t)(blocks ? blocks : 1));
        for (int b = 0; b < blocks; ++b) {
            const int first = b * CS_TAIL_BLOCK_FRAMES;
            const int end = first + CS_TAIL_BLOCK_FRAMES < job->frames ? first + CS_TAIL_BLOCK_FRAMES : job->frames;
            stats[b] = scanBlock(jobMix, first, end);
        }
        cs_tail_result result = selectNative(jobMix, stats, job);
        free(stats);
        int16_t* mono = malloc(sizeof(int16_t) * (size_t)(job->frames ? job->frames : 1));
        const int windows = (job->frames + window - 1) / window;
        MonoStats* monoStats = calloc((size_t)(windows ? windows : 1), sizeof(MonoStats));
        quantizeMono(jobMix, &result, window, mono, monoStats);
        selectTrim(monoStats, &result, &config);
        result.offset = offset;
        result.peak = 0;
        result.first = result.frames;
        result.last = -1;
        finalize(mono, 1, &result, packed ? packed + offset : mono, quality);
        offset += (size_t)result.dataFrames;
        results[j] = result;
        free(mono);
        free(monoStats);
        frameBase += (size_t)job->frames;
    }
    return offset;
}

/* orig/custom finishing (layoutPcm + finalizePcm with two channels). */
size_t oracle_finish_stereo(const int16_t* mix, const cs_plan* plans, int count, int quality,
                            cs_tail_result* results, int16_t* packed)
{
    size_t offset = 0;
    for (int j = 0; j < count; ++j) {
        cs_tail_result result;
        memset(&result, 0, sizeof result);
        result.frames = plans[j].frames;
        result.dataFrames = plans[j].frames;
        result.fade = plans[j].fade_frames;
        result.offset = offset;
        result.peak = 0;
        result.first = result.frames;
        result.last = -1;
        finalize(mix + 2 * offset, 2, &result, packed ? packed + 2 * offset : (int16_t*)(mix + 2 * offset), quality);
        offset += (size_t)result.dataFrames;
        results[j] = result;
    }
    return offset * 2;
}
