/*
 * ORACLE (test infrastructure, never shipped or measured): plain-C restatement of
 * the reference's quality gate, group volume matching and accepted-PCM packing,
 * src/cuda/quality.cu, for the checker.
 *
 * Input is a finished batch exactly as the tail stages leave it: packed PCM16
 * (mono for the natural tail, interleaved stereo otherwise) and one tail result
 * per job.  Every sum here is an integer sum (order-free) and every other step is
 * per job in the reference's own order, so the restatement is exact.
 * Only tests/ use it.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/claysampler_b200.h"

typedef unsigned long long Power;

/* monoPower (quality.cu:6-11): the mono sum of a frame, squared. */
static Power monoPower(const int16_t* pcm, int channels, long long frame)
{
    const int value = channels == 1 ? 2 * (int)pcm[frame] : (int)pcm[2 * frame] + (int)pcm[2 * frame + 1];
    return (Power)((long long)value * value);
}

/* bodyBlockStart (quality.cu:13-19): 250 ms windows restarting every 2 s. */
static int bodyBlockStart(int block, const cs_audio_config* c)
{
    const int chunk = 2 * c->rate, span = 5 * c->window;
    const int windows = (chunk + span - 1) / span;
    return (block / windows) * chunk + (block % windows) * span;
}

/* Renderer::bodyWindows (src/cuda/renderer.cpp:736-740). */
static int bodyWindows(int frames, const cs_audio_config* c)
{
    const int chunk = 2 * c->rate, span = 5 * c->window;
    return (frames / chunk) * ((chunk + span - 1) / span) + (frames % chunk + span - 1) / span;
}

/* level / percentile (quality.cu:93-104). */
static double level(Power power, int window)
{
    return power ? fmax(-120., 10 * log10((double)power / (window * 4294967296.))) : -120.;
}

static double percentile(const Power* sorted, int count, double fraction, int window)
{
    const double position = (count - 1) * fraction;
    const int first = (int)position;
    const double lower = level(sorted[first], window);
    return first + 1 < count ? lower + (level(sorted[first + 1], window) - lower) * (position - first) : lower;
}

/* The reference heap-sorts the onset powers (quality.cu:79-91, 139-148); any
 * ascending sort of integers gives the same array. */
static int ascending(const void* a, const void* b)
{
    const Power x = *(const Power*)a, y = *(const Power*)b;
    return x < y ? -1 : x > y;
}

static int imin(int a, int b) { return a < b ? a : b; }
static int imax(int a, int b) { return a > b ? a : b; }

/* measureBody + measureOnsets + summarizeAudio (quality.cu:21-77, 107-164) for one job. */
static void assessJob(const int16_t* pcm, int channels, const cs_plan* plan, const cs_audio_config* config,
                      cs_tail_result* result)
{
    if (result->status != CS_TAIL_OK)
        return;
    cs_audio_metrics* stats = &result->audio;
    const int body = config->enabled || plan->volume_group ? plan->body_frames : 0;
    const int windows = bodyWindows(body, config);
    const int16_t* audio = pcm + result->offset * (uint64_t)channels;
    Power* bodyPower = calloc((size_t)(windows ? windows : 1), sizeof(Power));
    for (int w = 0; w < windows; ++w) {
        const int end = imin(imin(body, result->dataFrames), bodyBlockStart(w + 1, config));
        for (int frame = bodyBlockStart(w, config); frame < end; ++frame)
            bodyPower[w] += monoPower(audio, channels, frame);
    }
    const int end = imin(result->frames, body);
    Power power = 0;
    int silent = 0, run = 0;
    for (int w = 0, first = 0; first < end; ++w) {
        const int next = imin(end, bodyBlockStart(w + 1, config));
        power += bodyPower[w];
        if (config->enabled) {
            if ((double)bodyPower[w] < (next - first) * config->silencePower) {
                silent += next - first;
                run += next - first;
                stats->longestSilence = imax(run, stats->longestSilence);
            } else {
                run = 0;
            }
        }
        first = next;
    }
    free(bodyPower);
    stats->bodyRms = body ? sqrt((double)power / body) * .5 : 0;
    if (!config->enabled)
        return;
    stats->measured = 1;
    stats->median = stats->quartile = -120;
    stats->silentFraction = (double)silent / imax(1, end);
    stats->clippedFraction = (double)stats->clipped / ((double)imax(1, result->frames) * channels);
    const int onsets = plan->onset_count;
    if (onsets) {
        Power* levels = calloc((size_t)onsets, sizeof(Power));
        for (int o = 0; o < onsets; ++o) {
            /* Five 50 ms windows from the onset; the loudest one counts. */
            for (int k = 0; k < 5; ++k) {
                const int first = plan->onsets[o] + k * config->window;
                const int stop = imin(first + config->window, result->dataFrames);
                Power p = 0;
                for (int frame = first; frame < stop; ++frame)
                    p += monoPower(audio, channels, frame);
                if (p > levels[o])
                    levels[o] = p;
            }
        }
        qsort(levels, (size_t)onsets, sizeof(Power), ascending);
        stats->median = percentile(levels, onsets, .5, config->window);
        stats->quartile = percentile(levels, onsets, .25, config->window);
        free(levels);
    }
    if (result->frames > config->maxFrames)
        result->status = CS_TAIL_AUDIO_DURATION;
    else if (!onsets || stats->median < config->minMedian || stats->quartile < config->minQuartile)
        result->status = CS_TAIL_QUIET_PERFORMANCE;
    else if (stats->silentFraction > config->maxSilentFraction || stats->longestSilence > config->maxSilentFrames)
        result->status = CS_TAIL_EXCESSIVE_SILENCE;
    else if (result->peak < config->minPeak)
        result->status = CS_TAIL_SILENT_AUDIO;
    else if (stats->clippedFraction > config->maxClippedFraction)
        result->status = CS_TAIL_CLIPPING;
    stats->verdict = result->status;
}

/* matchVolume (quality.cu:173-208) for members [first, end). */
static void matchGroup(cs_tail_result* results, int first, int end, int minimum)
{
    double desired = 0, safe = 1e30;
    int accepted = 0;
    for (int i = first; i < end; ++i) {
        cs_tail_result* result = &results[i];
        if (result->status != CS_TAIL_OK)
            continue;
        const double rms = result->audio.bodyRms;
        if (rms <= 0 || result->last < 0) {
            result->status = CS_TAIL_SILENT_BODY;
            continue;
        }
        desired += rms;
        const double ceiling = 32767 * .8912509381337456;    /* -1 dBFS */
        safe = fmin(safe, ceiling * rms / imax(1, result->peak));
        ++accepted;
    }
    const double target = fmin(desired / imax(1, accepted), safe);
    for (int i = first; i < end; ++i) {
        cs_tail_result* result = &results[i];
        if (result->status != CS_TAIL_OK)
            continue;
        if (accepted < minimum) {
            result->status = CS_TAIL_INCOMPLETE_GROUP;
        } else {
            result->audio.targetRms = target;
            result->audio.gain = target / result->audio.bodyRms;
        }
    }
}

/* layoutAccepted + packAccepted (quality.cu:211-280): drops rejected and silent
 * jobs from the PCM, applies group gains and re-measures gained jobs' peak and
 * audible range (each 1024-frame block merges its peak; audible range only from
 * blocks with an audible frame). */
static size_t packAccepted(const int16_t* source, int channels, const cs_plan* plans, int count,
                           cs_tail_result* results, int16_t* output)
{
    uint64_t offset = 0;
    for (int j = 0; j < count; ++j) {
        cs_tail_result* result = &results[j];
        const uint64_t sourceOffset = result->offset;
        if (result->status != CS_TAIL_OK || result->last < 0)
            result->dataFrames = 0;
        result->offset = offset;
        offset += (uint64_t)result->dataFrames;
        const double gain = result->audio.gain;
        if (gain > 0) {
            result->peak = 0;
            result->first = result->frames;
            result->last = -1;
        }
        const int16_t* input = source + sourceOffset * (uint64_t)channels;
        int16_t* pcm = output + result->offset * (uint64_t)channels;
        for (int first = 0; first < plans[j].frames; first += CS_TAIL_BLOCK_FRAMES) {
            const int end = imin(first + CS_TAIL_BLOCK_FRAMES, result->dataFrames);
            if (first >= end)
                break;
            int peak = 0, audibleFirst = result->frames, audibleLast = -1;
            for (int frame = first; frame < end; ++frame) {
                int framePeak = 0;
                for (int c = 0; c < channels; ++c) {
                    const size_t sample = (size_t)frame * channels + c;
                    const int16_t value = gain > 0 ? (int16_t)(int)nearbyint(input[sample] * gain) : input[sample];
                    pcm[sample] = value;
                    framePeak = imax(framePeak, abs((int)value));
                }
                peak = imax(peak, framePeak);
                if (framePeak > 3) {
                    audibleFirst = imin(audibleFirst, frame);
                    audibleLast = frame;
                }
            }
            if (gain > 0) {
                result->peak = imax(result->peak, peak);
                if (audibleLast >= 0) {
                    result->first = imin(result->first, audibleFirst);
                    result->last = imax(result->last, audibleLast);
                }
            }
        }
    }
    return (size_t)offset * channels;
}

/* The assessment of one finished batch as the reference renderer runs it when the
 * quality gate or group volume is on (renderer.cpp:1170-1180, 1143-1148, 1134-1141):
 * clipped-sample counts, body and onset levels, verdicts, group gains for the
 * volume groups the batch holds (runs of equal nonzero plan volume_group), then
 * the accepted PCM.  `results` holds the tail results on entry; `accepted`
 * receives the packed accepted PCM; returns its sample count. */
size_t oracle_assess(const int16_t* finished, int channels, const cs_plan* plans, int count,
                     const cs_audio_config* config, int group_minimum, cs_tail_result* results, int16_t* accepted)
{
    for (int j = 0; j < count; ++j) {
        cs_tail_result* result = &results[j];
        if (config->enabled) {
            /* finalizePcm's clipped count over the job's finished samples (tail.cu:262-285). */
            const int16_t* audio = finished + result->offset * (uint64_t)channels;
            int clipped = 0;
            for (long long s = 0; s < (long long)result->dataFrames * channels; ++s)
                clipped += abs((int)audio[s]) >= 32767;
            result->audio.clipped = clipped;
        }
        assessJob(finished, channels, &plans[j], config, result);
    }
    if (group_minimum > 0) {
        for (int first = 0, end; first < count; first = end) {
            end = first + 1;
            if (!plans[first].volume_group)
                continue;
            while (end < count && plans[end].volume_group == plans[first].volume_group)
                ++end;
            matchGroup(results, first, end, group_minimum);
        }
    }
    return packAccepted(finished, channels, plans, count, results, accepted);
}

/* The group step alone, for a group whose members were assessed in several
 * batches: matchVolume over results[0, count) then packAccepted of one batch's
 * slice [first, first + jobs) from its finished PCM. */
void oracle_match_group(cs_tail_result* results, int count, int group_minimum)
{
    matchGroup(results, 0, count, group_minimum);
}

size_t oracle_pack_accepted(const int16_t* source, int channels, const cs_plan* plans, int count,
                            cs_tail_result* results, int16_t* output)
{
    return packAccepted(source, channels, plans, count, results, output);
}
