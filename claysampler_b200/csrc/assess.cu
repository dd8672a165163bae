// Quality gate, group volume and accepted-PCM packing (sm_100a): the reference's
// src/cuda/quality.cu stages after finishing.
//
//  onsetKernel      one CTA of five warps per MIDI onset: each warp sums the mono
//                   power of one 50 ms window, the CTA keeps the loudest
//                   (measureOnsets, quality.cu:48-77).
//  summarizeKernel  one warp per job: body RMS and silence runs over the job's
//                   250 ms body windows (lanes take contiguous runs of windows and
//                   the runs are joined in order), onset percentiles by a warp radix
//                   select instead of the reference's serial heap sort, and the
//                   verdict (summarizeAudio, quality.cu:107-170).
//  matchKernel      one thread per volume group, members in order, so the mean is
//                   summed in the reference's order (matchVolume, quality.cu:173-208).
//  layoutAccepted   one warp: exclusive scan of accepted frames (quality.cu:211-232).
//  packAccepted     one CTA per 1024-frame block: gain, copy, and peak / audible range
//                   of gained jobs (quality.cu:234-280).
// Body power itself is summed inside the finishing pass (finalizeKernel).
#include "kernels.cuh"

namespace cs {
namespace {

constexpr unsigned kAll = 0xffffffffu;
constexpr int kSummaryWarps = 8;

template <class T>
__device__ __forceinline__ T warpSum(T value)
{
    #pragma unroll
    for (int d = 16; d; d >>= 1)
        value += __shfl_xor_sync(kAll, value, d);
    return value;
}

__device__ __forceinline__ int warpMax(int value)
{
    #pragma unroll
    for (int d = 16; d; d >>= 1)
        value = max(value, __shfl_xor_sync(kAll, value, d));
    return value;
}

__device__ __forceinline__ int warpMin(int value)
{
    #pragma unroll
    for (int d = 16; d; d >>= 1)
        value = min(value, __shfl_xor_sync(kAll, value, d));
    return value;
}

// Squared mono sum of one frame (monoPower, quality.cu:6-11).
template <int Channels>
__device__ __forceinline__ unsigned long long monoPower(const short* pcm, int frame)
{
    const int value = Channels == 1 ? 2 * int(pcm[frame]) : int(pcm[2 * frame]) + int(pcm[2 * frame + 1]);
    return (unsigned long long)((long long)value * value);
}

template <int Channels>
__global__ void __launch_bounds__(160) onsetKernel(AssessView a, const cs_tail_result* results, const short* pcm)
{
    __shared__ unsigned long long windows[5];
    const int onset = int(blockIdx.x);
    const cs_tail_result& result = results[a.onsetJob[onset]];
    if (result.status != CS_TAIL_OK)
        return;
    const int warp = int(threadIdx.x >> 5), lane = int(threadIdx.x & 31);
    const int first = a.onsets[onset] + warp * a.config.window;
    const int end = min(first + a.config.window, result.dataFrames);
    const short* audio = pcm + result.offset * Channels;
    unsigned long long power = 0;
    for (int frame = first + lane; frame < end; frame += 32)
        power += monoPower<Channels>(audio, frame);
    power = warpSum(power);
    if (!lane)
        windows[warp] = power;
    __syncthreads();
    if (threadIdx.x == 0)
        a.onsetPower[onset] = max(max(max(windows[0], windows[1]), max(windows[2], windows[3])), windows[4]);
}

// The k-th smallest (0-based) of `count` values: eight passes over 8-bit digits from
// the top, each narrowing the candidates to one histogram bin (one warp).
__device__ unsigned long long selectRank(const unsigned long long* values, int count, int k, unsigned* histogram)
{
    const int lane = int(threadIdx.x & 31);
    unsigned long long prefix = 0, mask = 0;
    for (int shift = 56; shift >= 0; shift -= 8) {
        for (int i = lane; i < 256; i += 32)
            histogram[i] = 0;
        __syncwarp();
        for (int i = lane; i < count; i += 32) {
            const unsigned long long value = values[i];
            if ((value & mask) == prefix)
                atomicAdd(histogram + ((value >> shift) & 255), 1u);
        }
        __syncwarp();
        unsigned local = 0;
        #pragma unroll
        for (int j = 0; j < 8; ++j)
            local += histogram[lane * 8 + j];
        unsigned inclusive = local;
        #pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const unsigned up = __shfl_up_sync(kAll, inclusive, d);
            if (lane >= d)
                inclusive += up;
        }
        const unsigned exclusive = inclusive - local;
        const unsigned owner = __ffs(__ballot_sync(kAll, unsigned(k) >= exclusive && unsigned(k) < inclusive)) - 1;
        int bin = 0, rest = 0;
        if (lane == int(owner)) {
            unsigned seen = exclusive;
            for (int j = 0; j < 8; ++j) {
                const unsigned n = histogram[lane * 8 + j];
                if (unsigned(k) < seen + n) {
                    bin = lane * 8 + j;
                    rest = k - int(seen);
                    break;
                }
                seen += n;
            }
        }
        bin = __shfl_sync(kAll, bin, int(owner));
        k = __shfl_sync(kAll, rest, int(owner));
        prefix |= (unsigned long long)bin << shift;
        mask |= 255ull << shift;
        __syncwarp();
    }
    return prefix;
}

__device__ double level(unsigned long long power, int window)
{
    return power ? fmax(-120., 10 * log10(double(power) / (window * 4294967296.))) : -120.;
}

// percentile (quality.cu:98-104) of the sorted onset powers.
__device__ double percentile(const unsigned long long* values, int count, double fraction, int window,
                             unsigned* histogram)
{
    const double position = (count - 1) * fraction;
    const int first = int(position);
    const double lower = level(selectRank(values, count, first, histogram), window);
    if (first + 1 >= count)
        return lower;
    return lower + (level(selectRank(values, count, first + 1, histogram), window) - lower) * (position - first);
}

template <int Channels>
__global__ void __launch_bounds__(kSummaryWarps * 32) summarizeKernel(AssessView a, cs_tail_result* results)
{
    __shared__ unsigned histograms[kSummaryWarps][256];
    const int warp = int(threadIdx.x >> 5), lane = int(threadIdx.x & 31);
    const int jobIndex = int(blockIdx.x) * kSummaryWarps + warp;
    if (jobIndex >= a.jobCount)
        return;
    cs_tail_result& result = results[jobIndex];
    if (result.status != CS_TAIL_OK)
        return;
    const AssessJob job = a.jobs[jobIndex];
    const cs_audio_config& config = a.config;
    const int end = min(result.frames, job.bodyFrames);
    const int windows = end > 0 ? a.body.windowOf(end - 1) + 1 : 0;
    // Lane `lane` takes windows [w0, w1): its power and silent frames, the silent
    // frames before its first loud window (`lead`, all of them when none is loud),
    // its longest inner silent run and the silent run it ends with.
    const int per = (windows + 31) / 32;
    const int w0 = min(windows, lane * per), w1 = min(windows, w0 + per);
    unsigned long long power = 0;
    int silent = 0, lead = 0, longest = 0, run = 0;
    bool loud = false;
    for (int w = w0; w < w1; ++w) {
        const int first = a.body.start(w), next = min(end, a.body.start(w + 1));
        const unsigned long long windowPower = a.bodyPower[job.bodyFirst + w];
        power += windowPower;
        if (config.enabled) {
            if (double(windowPower) < (next - first) * config.silencePower) {
                silent += next - first;
                run += next - first;
                longest = max(longest, run);
                if (!loud)
                    lead += next - first;
            } else {
                run = 0;
                loud = true;
            }
        }
    }
    power = warpSum(power);
    silent = warpSum(silent);
    // Join the lanes' runs in window order.
    int carry = 0, best = 0;
    for (int l = 0; l < 32; ++l) {
        const int laneLead = __shfl_sync(kAll, lead, l), laneLongest = __shfl_sync(kAll, longest, l);
        const int laneRun = __shfl_sync(kAll, run, l);
        const bool laneLoud = __shfl_sync(kAll, loud ? 1 : 0, l) != 0;
        if (!laneLoud) {
            carry += laneLead;
            best = max(best, carry);
        } else {
            best = max(best, max(carry + laneLead, laneLongest));
            carry = laneRun;
        }
    }
    cs_audio_metrics stats = result.audio;
    stats.longestSilence = max(stats.longestSilence, best);
    stats.bodyRms = job.bodyFrames ? sqrt(double(power) / job.bodyFrames) * .5 : 0;
    int status = result.status;
    if (config.enabled) {
        stats.measured = 1;
        stats.median = stats.quartile = -120;
        stats.silentFraction = double(silent) / max(1, end);
        stats.clippedFraction = double(stats.clipped) / (double(max(1, result.frames)) * Channels);
        if (job.onsetCount) {
            const unsigned long long* levels = a.onsetPower + job.onsetFirst;
            stats.median = percentile(levels, job.onsetCount, .5, config.window, histograms[warp]);
            stats.quartile = percentile(levels, job.onsetCount, .25, config.window, histograms[warp]);
        }
        if (result.frames > config.maxFrames)
            status = CS_TAIL_AUDIO_DURATION;
        else if (!job.onsetCount || stats.median < config.minMedian || stats.quartile < config.minQuartile)
            status = CS_TAIL_QUIET_PERFORMANCE;
        else if (stats.silentFraction > config.maxSilentFraction || stats.longestSilence > config.maxSilentFrames)
            status = CS_TAIL_EXCESSIVE_SILENCE;
        else if (result.peak < config.minPeak)
            status = CS_TAIL_SILENT_AUDIO;
        else if (stats.clippedFraction > config.maxClippedFraction)
            status = CS_TAIL_CLIPPING;
        stats.verdict = status;
    }
    if (lane == 0) {
        result.audio = stats;
        result.status = status;
    }
}

__global__ void matchKernel(const int2* groups, int count, int minimum, cs_tail_result* results)
{
    const int index = int(blockIdx.x * blockDim.x + threadIdx.x);
    if (index >= count)
        return;
    const int2 group = groups[index];
    double desired = 0, safe = 1e30;
    int accepted = 0;
    for (int i = group.x; i < group.y; ++i) {
        cs_tail_result& result = results[i];
        if (result.status != CS_TAIL_OK)
            continue;
        const double rms = result.audio.bodyRms;
        if (rms <= 0 || result.last < 0) {
            result.status = CS_TAIL_SILENT_BODY;
            continue;
        }
        desired += rms;
        constexpr double ceiling = 32767 * .8912509381337456;   // -1 dBFS
        safe = fmin(safe, ceiling * rms / max(1, result.peak));
        ++accepted;
    }
    const double target = fmin(desired / max(1, accepted), safe);
    for (int i = group.x; i < group.y; ++i) {
        cs_tail_result& result = results[i];
        if (result.status != CS_TAIL_OK)
            continue;
        if (accepted < minimum) {
            result.status = CS_TAIL_INCOMPLETE_GROUP;
        } else {
            result.audio.targetRms = target;
            result.audio.gain = target / result.audio.bodyRms;
        }
    }
}

__global__ void layoutAcceptedKernel(PackView p)
{
    const int lane = int(threadIdx.x);
    unsigned long long carry = 0;
    for (int base = 0; base < p.jobCount; base += 32) {
        const int i = base + lane;
        unsigned long long own = 0;
        if (i < p.jobCount) {
            const cs_tail_result& result = p.results[i];
            if (result.status == CS_TAIL_OK && result.last >= 0)
                own = (unsigned long long)result.dataFrames;
        }
        unsigned long long scan = own;
        #pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const unsigned long long up = __shfl_up_sync(kAll, scan, d);
            if (lane >= d)
                scan += up;
        }
        if (i < p.jobCount) {
            cs_tail_result& result = p.results[i];
            p.sourceOffset[i] = result.offset;
            result.dataFrames = int(own);
            result.offset = carry + scan - own;
            if (result.audio.gain > 0) {
                result.peak = 0;
                result.first = result.frames;
                result.last = -1;
            }
        }
        carry += __shfl_sync(kAll, scan, 31);
    }
}

template <int Channels>
__global__ void __launch_bounds__(128) packAcceptedKernel(PackView p)
{
    __shared__ int reduce[3][4];
    const int block = int(blockIdx.x);
    const int jobIndex = p.blockJob[block];
    cs_tail_result& result = p.results[jobIndex];
    const int first = (block - p.jobBlockFirst[jobIndex]) * kBlockFrames;
    const int end = min(first + kBlockFrames, result.dataFrames);
    if (first >= end)
        return;
    const double gain = result.audio.gain;
    const int frames = result.frames;
    const short* input = p.source + p.sourceOffset[jobIndex] * Channels;
    short* output = p.output + result.offset * Channels;
    int peak = 0, audibleFirst = frames, audibleLast = -1;
    for (int frame = first + int(threadIdx.x); frame < end; frame += blockDim.x) {
        int framePeak = 0;
        #pragma unroll
        for (int c = 0; c < Channels; ++c) {
            const size_t sample = size_t(frame) * Channels + c;
            const short value = gain > 0 ? short(__double2int_rn(input[sample] * gain)) : input[sample];
            output[sample] = value;
            framePeak = max(framePeak, abs(int(value)));
        }
        peak = max(peak, framePeak);
        if (framePeak > 3) {
            audibleFirst = min(audibleFirst, frame);
            audibleLast = frame;
        }
    }
    if (!(gain > 0))                     // uniform across the block
        return;
    const int warp = int(threadIdx.x >> 5), lane = int(threadIdx.x & 31);
    peak = warpMax(peak);
    audibleFirst = warpMin(audibleFirst);
    audibleLast = warpMax(audibleLast);
    if (!lane) {
        reduce[0][warp] = peak;
        reduce[1][warp] = audibleFirst;
        reduce[2][warp] = audibleLast;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < 4; ++w) {
            peak = max(peak, reduce[0][w]);
            audibleFirst = min(audibleFirst, reduce[1][w]);
            audibleLast = max(audibleLast, reduce[2][w]);
        }
        atomicMax(&result.peak, peak);
        if (audibleLast >= 0) {
            atomicMin(&result.first, audibleFirst);
            atomicMax(&result.last, audibleLast);
        }
    }
}

} // namespace

int launchMeasure(const AssessView& a, cs_tail_result* results, const short* pcm, bool natural, cudaStream_t stream)
{
    int launches = 0;
    if (a.config.enabled && a.onsetCount) {
        if (natural)
            onsetKernel<1><<<a.onsetCount, 160, 0, stream>>>(a, results, pcm);
        else
            onsetKernel<2><<<a.onsetCount, 160, 0, stream>>>(a, results, pcm);
        ++launches;
    }
    if (a.jobCount) {
        const int grid = (a.jobCount + kSummaryWarps - 1) / kSummaryWarps;
        if (natural)
            summarizeKernel<1><<<grid, kSummaryWarps * 32, 0, stream>>>(a, results);
        else
            summarizeKernel<2><<<grid, kSummaryWarps * 32, 0, stream>>>(a, results);
        ++launches;
    }
    return launches;
}

int launchMatch(const int2* groups, int count, int minimum, cs_tail_result* results, cudaStream_t stream)
{
    if (!count)
        return 0;
    matchKernel<<<(count + 31) / 32, 32, 0, stream>>>(groups, count, minimum, results);
    return 1;
}

int launchPack(const PackView& p, bool natural, cudaStream_t stream)
{
    if (!p.jobCount)
        return 0;
    layoutAcceptedKernel<<<1, 32, 0, stream>>>(p);
    if (!p.blockCount)
        return 1;
    if (natural)
        packAcceptedKernel<1><<<p.blockCount, 128, 0, stream>>>(p);
    else
        packAcceptedKernel<2><<<p.blockCount, 128, 0, stream>>>(p);
    return 2;
}

} // namespace cs
