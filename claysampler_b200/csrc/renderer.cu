// Host orchestration and C ABI of the B200 renderer.
//
// A batch of plans becomes one device arena holding the spans, control points,
// modulation bindings, per-job records, mix tiles, the float mix and the finishing
// buffers.  Render windows (cs_render_window, cs_submit / cs_poll) keep up to four
// batches in flight, each on a stream lane with its own arena and page-locked
// staging and download buffers; their kernels run in batch order on one compute
// stream, and within a render window the shared voice sources are pooled across
// its batches.  Voice chains that need filter or pitch storage write it to a scratch
// region; when that storage exceeds the scratch budget the job timeline is cut into
// 1024-frame-aligned segments and chain state (filter history, coefficient
// smoothing, pitch phase) carries across them in ChainState, as the reference's
// segmented synthesis does (src/cuda/renderer.cpp:864-932, render.cu:228-265,345-446).
#include "host_copy.hpp"
#include "kernels.cuh"
#include "plan_blob.hpp"

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <future>
#include <limits>
#include <memory>
#include <tuple>
#include <map>
#include <numeric>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

namespace cs {
namespace {

thread_local std::string lastError;

struct CudaError : std::runtime_error {
    cudaError_t code;
    CudaError(cudaError_t status, const char* what)
        : std::runtime_error(std::string(what) + ": " + cudaGetErrorString(status)), code(status) {}
};

void check(cudaError_t status, const char* what)
{
    if (status != cudaSuccess)
        throw CudaError(status, what);
}

size_t align256(size_t value) { return (value + 255) & ~size_t(255); }

struct Layout {
    size_t bytes = 0;
    size_t add(size_t size)
    {
        const size_t offset = align256(bytes);
        bytes = offset + size;
        return offset;
    }
};

// The reference's BatchIndex::append (src/cuda/renderer.cpp:390-460) restated for
// this renderer's layout: rebased control and modulation offsets, voice chains
// linked by nextFilteredSpan, and per job the inputs from which tileIndexKernel
// builds the 256-frame tiles' span-ordered voice lists on the device.
struct HostBatch {
    std::vector<cs_voice_span> voices;
    // Control points stay in the callers' plans; each plan's points are copied once,
    // straight into the pinned upload buffer.
    std::vector<std::pair<const cs_control_point*, size_t>> pointSources;
    size_t pointCount = 0;
    std::vector<cs_voice_modulation> modulation;
    std::vector<JobInfo> jobs;
    // The mix tiles' voice lists are built on the device (tileIndexKernel) from
    // each job's spans and index base, one unit per (job, chunk of tiles).
    std::vector<JobSpans> jobSpans;
    std::vector<int2> indexUnits;
    size_t tileCount = 0, indexCount = 0;
    std::vector<int> blockJob, windowJob, chainHeads, pitchHeads, jobBlockFirst;
    size_t frames = 0;
    int blocks = 0, windows = 0, lastFrame = 0;
    // Quality gate / group volume inputs (src/cuda/renderer.cpp:801-842).
    std::vector<AssessJob> assess;
    std::vector<int> onsets, onsetJob;
    std::vector<uint64_t> volumeGroups;
    int bodyWindows = 0;

    // Stages `count` plans.  `assessing`: the quality gate or group volume is on;
    // `quality`: the gate is.  A sequential pass checks the plans and sizes every
    // job's share of each array; the jobs are then filled in parallel.
    void build(const cs_plan* plans, size_t count, int window, bool natural, bool assessing, bool quality,
               const BodyGeometry& body, WorkerPool& pool)
    {
        struct Share {
            size_t voice, modulation, tile, index, point, onset, block, window, frame;
            int bodyWindow;
        };
        std::vector<Share> at(count + 1);
        Share next{};
        for (size_t j = 0; j < count; ++j) {
            const cs_plan& plan = plans[j];
            if (plan.track_count < 3)
                throw std::runtime_error("a plan needs its CC7, CC11 and CC10 tracks");
            at[j] = next;
            size_t entries = 0;
            for (int k = 0; k < plan.span_count; ++k) {
                const auto& span = plan.spans[k];
                if (span.begin < 0 || span.end > plan.frames || span.begin >= span.end)
                    throw std::runtime_error("span outside its job's frames");
                if (span.filterTrack >= plan.filter_tracks)
                    throw std::runtime_error("span filter track outside the plan's filter_tracks");
                entries += size_t((span.end - 1) / kTileFrames - span.begin / kTileFrames + 1);
            }
            const int onsetCount = assessing && quality ? plan.onset_count : 0;
            for (int k = 0; k < onsetCount; ++k)
                if (plan.onsets[k] < 0)
                    throw std::runtime_error("negative onset frame");
            const int64_t points = plan.track_offsets[plan.track_count] - plan.track_offsets[0];
            next.voice += size_t(plan.span_count);
            next.modulation += size_t(plan.modulation_count);
            next.tile += size_t((plan.frames + kTileFrames - 1) / kTileFrames);
            next.index += entries;
            next.point += size_t(points);
            next.onset += size_t(onsetCount);
            next.block += size_t((plan.frames + kBlockFrames - 1) / kBlockFrames);
            next.window += natural ? size_t((plan.frames + window - 1) / window) : 0;
            next.frame += size_t(plan.frames);
            if (assessing)
                next.bodyWindow += body.windows(quality || plan.volume_group ? plan.body_frames : 0);
        }
        at[count] = next;
        if (next.point > size_t(INT32_MAX) || next.voice > size_t(INT32_MAX) || next.index > size_t(INT32_MAX) ||
            next.block > size_t(INT32_MAX) || next.window > size_t(INT32_MAX) || next.tile > size_t(INT32_MAX))
            throw std::runtime_error("batch too large for 32-bit indices");
        voices.resize(next.voice);
        modulation.resize(next.modulation);
        tileCount = next.tile;
        indexCount = next.index;
        jobSpans.resize(count);
        indexUnits.clear();
        for (size_t j = 0; j < count; ++j) {
            const int chunks = int((at[j + 1].tile - at[j].tile + kIndexChunkTiles - 1) / kIndexChunkTiles);
            for (int c = 0; c < chunks; ++c)
                indexUnits.push_back(make_int2(int(j), c));
        }
        blockJob.resize(next.block);
        windowJob.resize(next.window);
        jobs.resize(count);
        jobBlockFirst.resize(count);
        volumeGroups.resize(count);
        pointSources.resize(count);
        if (assessing) {
            assess.resize(count);
            onsets.resize(next.onset);
            onsetJob.resize(next.onset);
        }
        std::vector<std::vector<int>> heads(count), pitch(count);
        pool.run(count, [&](size_t j) {
            const cs_plan& plan = plans[j];
            const Share& base = at[j];
            JobInfo& job = jobs[j];
            job = JobInfo{};
            job.offset = base.frame;
            job.frames = plan.frames;
            job.musicEnd = plan.music_end;
            job.limit = plan.limit;
            job.fade = plan.fade_frames;
            job.blockFirst = int(base.block);
            job.windowFirst = int(base.window);
            job.tileFirst = int(base.tile);
            // Track offsets rebased onto the batch's point array.
            std::vector<int> pointOffsets(size_t(plan.track_count) + 1);
            for (int i = 0; i <= plan.track_count; ++i)
                pointOffsets[size_t(i)] = int(base.point + size_t(plan.track_offsets[i] - plan.track_offsets[0]));
            pointSources[j] = {plan.points + plan.track_offsets[0], at[j + 1].point - base.point};
            for (int i = 0; i < 4; ++i)
                job.tracks[i] = pointOffsets[size_t(i)];
            for (int m = 0; m < plan.modulation_count; ++m) {
                cs_voice_modulation binding = plan.modulation[m];
                if (binding.first >= 0) {
                    binding.last = pointOffsets[size_t(binding.first) + 1];
                    binding.first = pointOffsets[size_t(binding.first)];
                }
                if (binding.shapeFirst >= 0) {
                    binding.shapeLast = pointOffsets[size_t(binding.shapeFirst) + 1];
                    binding.shapeFirst = pointOffsets[size_t(binding.shapeFirst)];
                }
                modulation[base.modulation + size_t(m)] = binding;
            }
            jobSpans[j] = JobSpans{int(base.voice), plan.span_count, int(base.index), 0};
            std::vector<int> chainTail(size_t(plan.filter_tracks), -1);
            for (int k = 0; k < plan.span_count; ++k) {
                cs_voice_span voice = plan.spans[k];
                const int index = int(base.voice) + k;
                voice.firstModulation += int(base.modulation);
                if (voice.filterTrack >= 0) {
                    int& tail = chainTail[size_t(voice.filterTrack)];
                    if (tail < 0) {
                        heads[j].push_back(index);
                        if (voice.variablePitch)
                            pitch[j].push_back(index);
                    } else {
                        voices[size_t(tail)].nextFilteredSpan = index;
                    }
                    tail = index;
                    voice.nextFilteredSpan = -1;
                    for (int i = 0; i < 4; ++i)
                        voice.filterControls[i] = pointOffsets[size_t(i)];
                }
                voices[size_t(index)] = voice;
            }
            if (assessing) {
                const int bodyFrames = quality || plan.volume_group ? plan.body_frames : 0;
                const int onsetCount = int(at[j + 1].onset - base.onset);
                assess[j] = {bodyFrames, base.bodyWindow, int(base.onset), onsetCount};
                for (int i = 0; i < onsetCount; ++i) {
                    onsets[base.onset + size_t(i)] = plan.onsets[i];
                    onsetJob[base.onset + size_t(i)] = int(j);
                }
            }
            volumeGroups[j] = plan.volume_group;
            jobBlockFirst[j] = int(base.block);
            for (size_t b = base.block; b < at[j + 1].block; ++b)
                blockJob[b] = int(j);
            for (size_t w = base.window; w < at[j + 1].window; ++w)
                windowJob[w] = int(j);
        });
        for (size_t j = 0; j < count; ++j) {
            chainHeads.insert(chainHeads.end(), heads[j].begin(), heads[j].end());
            pitchHeads.insert(pitchHeads.end(), pitch[j].begin(), pitch[j].end());
            lastFrame = std::max(lastFrame, plans[j].frames);
        }
        pointCount = next.point;
        frames = next.frame;
        blocks = int(next.block);
        windows = int(next.window);
        bodyWindows = next.bodyWindow;
    }
};

struct SegmentPlan {
    int first, end;
    size_t scratchFloats, phaseFrames;
    size_t chainFirst, chainCount, simpleFirst, simpleCount, pitchFirst, pitchCount, blockFirst, blockCount;
    size_t tileFirst, tileCount;
    // The longest single-slot chains and their source tiles come first, in lead
    // tiers of decreasing length: a tier's recurrences start as soon as its sources
    // are rendered, beside the sources of the later tiers and the rest.  Tier k
    // holds the chains of at least 1/2^(k+1) of the longest chain's frames;
    // leadChains[k] / leadTiles[k] are its chain and source-tile counts (0: none).
    int leadTiers;
    size_t leadChains[kLeadTiers], leadTiles[kLeadTiers];
};

// Host side of a staged batch: segment boundaries and the per-segment arrays.
struct SegmentTables {
    std::vector<SegmentPlan> segments;
    std::vector<uint64_t> scratchOffset, phaseOffset, targetOffset;   // segments x voices
    std::vector<int> chains, simple, pitch, blocks;
    std::vector<int4> tileRuns;         // (span, first frame, end frame, first tile) per span
    size_t tileCount = 0;               // source tiles of all segments
    size_t scratchBytes = 0;
    size_t fullScratchBytes = 0;        // chain storage of the whole timeline in one segment
};

// A chain runs on the one-recurrence-per-lane kernel when every span filters
// through at most one of the two main slots, and always the same one.
bool singleSlotChain(const HostBatch& batch, int head)
{
    int slot = -1, type = CS_FILTER_NONE;
    for (int span = head; span >= 0; span = batch.voices[size_t(span)].nextFilteredSpan) {
        const auto& v = batch.voices[size_t(span)];
        int spanSlot = -1;
        for (int f = 0; f < CS_FILTER_SLOTS; ++f) {
            if (v.filters[f].type == CS_FILTER_NONE)
                continue;
            if (f >= 2 || spanSlot >= 0)
                return false;
            spanSlot = f;
        }
        if (spanSlot >= 0) {
            if (slot >= 0 && (slot != spanSlot || v.filters[spanSlot].type != type))
                return false;
            slot = spanSlot;
            type = v.filters[spanSlot].type;
            if (type == CS_FILTER_PEAK)
                return false;
        }
    }
    return true;
}

// filterMoves (render.cu:370-375) on the host.
bool spanMoves(const HostBatch& batch, const cs_voice_span& v)
{
    bool moving = v.activeEnvelope[0] != 0;
    for (int j = v.firstModulation; j < v.firstModulation + v.modulationCount; ++j) {
        const int target = batch.modulation[size_t(j)].target;
        moving |= (target >= CS_MOD_CUTOFF && target <= CS_MOD_RESONANCE2) || target == CS_MOD_FILEG_DEPTH ||
            target >= CS_MOD_EQ1_FREQUENCY;
    }
    return moving;
}

size_t scratchBytesOf(size_t floats, size_t phases) { return align256(floats * sizeof(float)) + phases * sizeof(double); }

size_t alignFloats(size_t floats) { return (floats + 3) & ~size_t(3); }

// Cuts [0, lastFrame) at 1024-frame boundaries so that each segment's chain
// storage fits `budget` (one block per segment at least), then lays out every
// segment's storage: per span its source frames (16-byte aligned) and, for
// single-slot chains, its filter targets (every frame when the filter moves, the
// first frame of the chain otherwise).
SegmentTables planSegments(const HostBatch& batch, size_t budget)
{
    SegmentTables t;
    const size_t voiceCount = batch.voices.size();
    // Chain membership and kind of every chain span.
    std::vector<int> chainOf(voiceCount, -1);
    std::vector<char> simple(voiceCount, 0), moving(voiceCount, 0), head(voiceCount, 0);
    for (int h : batch.chainHeads) {
        const bool single = singleSlotChain(batch, h);
        head[size_t(h)] = 1;
        for (int span = h; span >= 0; span = batch.voices[size_t(span)].nextFilteredSpan) {
            chainOf[size_t(span)] = h;
            simple[size_t(span)] = single;
            moving[size_t(span)] = spanMoves(batch, batch.voices[size_t(span)]);
        }
    }
    const auto hasFilter = [&](const cs_voice_span& v) {
        for (const auto& f : v.filters)
            if (f.type != CS_FILTER_NONE)
                return true;
        return false;
    };
    const auto targetFloats = [&](size_t v, int frames) -> size_t {
        if (!simple[v] || !hasFilter(batch.voices[v]))
            return 0;
        if (moving[v])
            return size_t((frames + kRecChunkFrames - 1) / kRecChunkFrames) * 3 * kRecChunkFrames;
        return head[v] ? 4 : 0;
    };
    const int lastFrame = batch.lastFrame;
    const int blocks = (lastFrame + kBlockFrames - 1) / kBlockFrames;
    // Per-block storage demand, via spans' block overlaps (slack for alignment): the
    // partial first and last blocks of a span directly, its full blocks through
    // difference arrays.
    std::vector<long long> floatsPerBlock(size_t(blocks) + 1, 0), phasesPerBlock(size_t(blocks) + 1, 0);
    std::vector<long long> fullFloats(size_t(blocks) + 1, 0), fullPhases(size_t(blocks) + 1, 0);
    for (size_t vi = 0; vi < voiceCount; ++vi) {
        const auto& v = batch.voices[vi];
        if (v.filterTrack < 0)
            continue;
        const auto add = [&](int b, int frames) {
            floatsPerBlock[size_t(b)] += (long long)frames * v.channels + 8 + (long long)targetFloats(vi, frames);
            if (v.variablePitch)
                phasesPerBlock[size_t(b)] += frames;
        };
        const int first = v.begin / kBlockFrames, last = (v.end - 1) / kBlockFrames;
        if (first == last) {
            add(first, v.end - v.begin);
            continue;
        }
        add(first, (first + 1) * kBlockFrames - v.begin);
        add(last, v.end - last * kBlockFrames);
        if (last - first > 1) {
            const long long full = (long long)kBlockFrames * v.channels + 8 + (long long)targetFloats(vi, kBlockFrames);
            fullFloats[size_t(first + 1)] += full;
            fullFloats[size_t(last)] -= full;
            if (v.variablePitch) {
                fullPhases[size_t(first + 1)] += kBlockFrames;
                fullPhases[size_t(last)] -= kBlockFrames;
            }
        }
    }
    for (long long b = 0, floatsRun = 0, phasesRun = 0; b < blocks; ++b) {
        floatsRun += fullFloats[size_t(b)];
        phasesRun += fullPhases[size_t(b)];
        floatsPerBlock[size_t(b)] += floatsRun;
        phasesPerBlock[size_t(b)] += phasesRun;
    }

    {
        size_t floats = 0, phases = 0;
        for (int b = 0; b < blocks; ++b) {
            floats += size_t(floatsPerBlock[size_t(b)]);
            phases += size_t(phasesPerBlock[size_t(b)]);
        }
        t.fullScratchBytes = scratchBytesOf(floats, phases);
    }
    std::vector<std::pair<int, int>> ranges;
    for (int b = 0; b < blocks;) {
        size_t floats = 0, phases = 0;
        int e = b;
        while (e < blocks) {
            const size_t nf = floats + size_t(floatsPerBlock[size_t(e)]);
            const size_t np = phases + size_t(phasesPerBlock[size_t(e)]);
            if (e > b && scratchBytesOf(nf, np) > budget)
                break;
            floats = nf;
            phases = np;
            ++e;
        }
        ranges.emplace_back(b * kBlockFrames, std::min(lastFrame, e * kBlockFrames));
        b = e;
    }
    if (ranges.empty())
        ranges.emplace_back(0, 0);
    t.scratchOffset.assign(voiceCount * ranges.size(), 0);
    t.phaseOffset.assign(voiceCount * ranges.size(), 0);
    t.targetOffset.assign(voiceCount * ranges.size(), kNoTargets);
    for (size_t si = 0; si < ranges.size(); ++si) {
        SegmentPlan seg{};
        seg.first = ranges[si].first;
        seg.end = ranges[si].second;
        size_t floats = 0, phases = 0;
        std::vector<size_t> targetNeed(voiceCount, 0);
        for (size_t v = 0; v < voiceCount; ++v) {
            const auto& voice = batch.voices[v];
            if (voice.filterTrack < 0)
                continue;
            const int frames = std::max(0, std::min(voice.end, seg.end) - std::max(voice.begin, seg.first));
            t.scratchOffset[si * voiceCount + v] = floats;
            t.phaseOffset[si * voiceCount + v] = phases;
            floats = alignFloats(floats + size_t(frames) * size_t(voice.channels));
            if (voice.variablePitch)
                phases += size_t(frames);
            if (frames > 0)
                targetNeed[v] = targetFloats(v, frames);
        }
        for (size_t v = 0; v < voiceCount; ++v) {
            if (!targetNeed[v])
                continue;
            t.targetOffset[si * voiceCount + v] = floats;
            floats += targetNeed[v];
        }
        seg.scratchFloats = floats;
        seg.phaseFrames = phases;
        t.scratchBytes = std::max(t.scratchBytes, scratchBytesOf(floats, phases));
        const auto active = [&](int h) {
            for (int span = h; span >= 0; span = batch.voices[size_t(span)].nextFilteredSpan) {
                const auto& v = batch.voices[size_t(span)];
                if (v.begin >= seg.end)
                    break;
                if (v.end > seg.first)
                    return true;
            }
            return false;
        };
        seg.chainFirst = t.chains.size();
        seg.tileFirst = t.tileCount;
        std::vector<std::pair<long long, int>> simpleChains;
        const auto framesIn = [&](const cs_voice_span& v) {
            return std::max(0, std::min(v.end, seg.end) - std::max(v.begin, seg.first));
        };
        for (int h : batch.chainHeads) {
            if (!active(h))
                continue;
            if (!simple[size_t(h)]) {
                t.chains.push_back(h);
                continue;
            }
            long long frames = 0;
            for (int span = h; span >= 0; span = batch.voices[size_t(span)].nextFilteredSpan)
                frames += framesIn(batch.voices[size_t(span)]);
            simpleChains.emplace_back(-frames, h);
        }
        seg.chainCount = t.chains.size() - seg.chainFirst;
        const auto simpleChains0 = simpleChains;      // plan order
        // Longest recurrences first: neighbouring lanes then run similar lengths.
        std::stable_sort(simpleChains.begin(), simpleChains.end(),
                         [](const auto& x, const auto& y) { return x.first < y.first; });
        // Lead tiers: tier k takes the chains of at least 1/2^(k+1) of the longest
        // chain's frames, in whole recurrence CTAs; the rest's recurrences then run
        // after all sources and are at most 1/2^kLeadTiers as long as the longest.
        // A tier that would take every remaining chain is left to the rest.
        seg.leadTiers = 0;
        std::vector<unsigned char> tierOf(voiceCount, kLeadTiers);
        size_t taken = 0;
        if (!simpleChains.empty()) {
            const long long longest = -simpleChains.front().first;
            for (int k = 0; k < kLeadTiers; ++k) {
                size_t end = taken;
                while (end < simpleChains.size() && (-simpleChains[end].first << (k + 1)) >= longest)
                    ++end;
                end = (end + kRecChainsPerCta - 1) / kRecChainsPerCta * kRecChainsPerCta;
                if (end >= simpleChains.size())
                    break;
                if (end == taken)
                    continue;
                for (size_t c = taken; c < end; ++c)
                    tierOf[size_t(simpleChains[c].second)] = static_cast<unsigned char>(seg.leadTiers);
                seg.leadChains[seg.leadTiers++] = end - taken;
                taken = end;
            }
        }
        // Source tiles: tier by tier, then the rest, each group in plan order
        // (neighbouring tiles then read neighbouring samples and tracks).
        for (int group = 0; group <= seg.leadTiers; ++group) {
            const size_t groupFirst = t.tileCount;
            const int tier = group < seg.leadTiers ? group : kLeadTiers;
            for (const auto& item : simpleChains0) {
                const int h = item.second;
                if (tierOf[size_t(h)] != tier)
                    continue;
                for (int span = h; span >= 0; span = batch.voices[size_t(span)].nextFilteredSpan) {
                    const auto& v = batch.voices[size_t(span)];
                    const int lo = std::max(v.begin, seg.first), hi = std::min(v.end, seg.end);
                    if (lo < hi) {
                        t.tileRuns.push_back(make_int4(span, lo, hi, int(t.tileCount)));
                        t.tileCount += size_t(hi - lo + kSourceTile - 1) / kSourceTile;
                    }
                }
            }
            if (group < seg.leadTiers)
                seg.leadTiles[group] = t.tileCount - groupFirst;
        }
        seg.tileCount = t.tileCount - seg.tileFirst;
        if (t.tileCount > size_t(INT32_MAX))
            throw std::runtime_error("too many source tiles in one batch");
        seg.simpleFirst = t.simple.size();
        for (const auto& item : simpleChains)
            t.simple.push_back(item.second);
        seg.simpleCount = t.simple.size() - seg.simpleFirst;
        seg.pitchFirst = t.pitch.size();
        for (int h : batch.pitchHeads)
            if (active(h))
                t.pitch.push_back(h);
        seg.pitchCount = t.pitch.size() - seg.pitchFirst;
        seg.blockFirst = t.blocks.size();
        for (const auto& job : batch.jobs) {
            const int jobBlocks = (job.frames + kBlockFrames - 1) / kBlockFrames;
            for (int b = seg.first / kBlockFrames; b < std::min(jobBlocks, (seg.end + kBlockFrames - 1) / kBlockFrames); ++b)
                t.blocks.push_back(job.blockFirst + b);
        }
        seg.blockCount = t.blocks.size() - seg.blockFirst;
        t.segments.push_back(seg);
    }
    return t;
}

// Shared voice sources: voices rendered inline (no filter chain) that play the
// same sample from the same position at the same step, with the same loop, loop
// crossfade and pitch ramp, have the same resampled source at every elapsed frame
// (render.cu:63-100 reads nothing else), so a batch renders it once and the mix
// reads it for each of them.  The audio is unchanged: the source is the same
// function of the same doubles.  Generators and variable-pitch voices stay inline.
struct WindowSource;

struct SharedPlan {
    std::vector<SharedSource> sources;
    // Render windows: the sources sit in the window's pool (offsets are pool
    // floats), and `claims` are the window sources this batch renders first.
    bool pooled = false;
    std::vector<WindowSource*> claims;
    std::vector<SharedRef> refs;        // per voice; empty when nothing is shared
    std::vector<int4> runs;             // (source, 0, frames, first tile) for tile expansion
    size_t tiles = 0, floats = 0;
    long long sharedVoiceFrames = 0;    // voice frames that read a shared source
    // Channel-frames that run the 48-tap sinc (step or pitch ramp away from 1):
    // rendered in the shared sources, and of the voices that read them instead.
    long long sincFloats = 0, sincVoiceFloats = 0;
};

bool resamples(const cs_voice_span& v) { return v.step != 1.0 || v.pitchSlope != 0; }

// The first elapsed frame at which a voice without loop or pitch ramp is past
// its sample's end in the device's double arithmetic, position + elapsed x step,
// whether the compiler fuses the multiply-add or not (the frame both forms put
// past the end); every later frame is past it as well.  The frames before it are
// rendered into the shared source, so a frame one form still finds inside the
// sample is never dropped.
long long silentFrom(const cs_voice_span& v)
{
    const double span = double(v.sourceEnd) - v.position;
    long long e = std::max<long long>(0, (long long)std::floor(span / v.step) - 2);
    for (;;) {
        const double distance = double(e);
        const double product = distance * v.step;
        const double separate = v.position + product;
        const double fused = std::fma(distance, v.step, v.position);
        if (separate >= double(v.sourceEnd) && fused >= double(v.sourceEnd))
            return e;
        ++e;
    }
}

// What a voice's source signal depends on (render.cu:63-100): equal keys give
// the same source at every elapsed frame.
struct SourceKey {
    uint64_t sample;
    double position, step, slope;
    int channels, sourceEnd, loopFirst, loopEnd, loopCrossfade;
    bool operator==(const SourceKey& o) const
    {
        return sample == o.sample && position == o.position && step == o.step && slope == o.slope &&
            channels == o.channels && sourceEnd == o.sourceEnd && loopFirst == o.loopFirst &&
            loopEnd == o.loopEnd && loopCrossfade == o.loopCrossfade;
    }
};

struct SourceKeyHash {
    size_t operator()(const SourceKey& k) const
    {
        uint64_t h = 0x9e3779b97f4a7c15ull;
        const auto mix = [&h](uint64_t v) { h = (h ^ v) * 0x100000001b3ull; h ^= h >> 29; };
        uint64_t bits;
        mix(k.sample);
        std::memcpy(&bits, &k.position, 8); mix(bits);
        std::memcpy(&bits, &k.step, 8); mix(bits);
        std::memcpy(&bits, &k.slope, 8); mix(bits);
        mix(uint64_t(uint32_t(k.channels)) << 32 | uint32_t(k.sourceEnd));
        mix(uint64_t(uint32_t(k.loopFirst)) << 32 | uint32_t(k.loopEnd));
        mix(uint64_t(uint32_t(k.loopCrossfade)));
        return size_t(h);
    }
};

// Whether a voice's source can be shared, its key, and the source frames it
// needs (to its span's end, or to the frame its source falls silent).
bool shareable(const cs_voice_span& v)
{
    return v.filterTrack < 0 && v.generator == CS_GEN_NONE && !v.variablePitch && v.end > v.begin &&
        v.channels >= 1 && v.channels <= 2;
}

SourceKey sourceKeyOf(const cs_voice_span& v)
{
    return SourceKey{v.sample, v.position, v.step, v.pitchSlope, v.channels, v.sourceEnd, v.loopFirst, v.loopEnd,
                     v.loopCrossfade};
}

long long sourceFramesOf(const cs_voice_span& v)
{
    long long frames = v.end - v.begin;
    if (v.loopEnd <= 0 && v.pitchSlope == 0 && v.step > 0)
        frames = std::min(frames, silentFrom(v));
    return frames;
}

// The shared sources of one render window: every source the window's voices
// play, at the longest length any of them needs, laid out in one device pool.  The first batch that plays a source renders it there (batches
// run their kernels in launch order on one stream), and later batches read it.
struct WindowSource {
    long long offset = 0;               // floats into the pool
    int frames = 0, channels = 0, users = 0;
    bool rendered = false;              // a launched batch renders it
    bool claimed = false;               // the batch being planned renders it
};

struct WindowSources {
    std::unordered_map<SourceKey, WindowSource, SourceKeyHash> map;
    size_t floats = 0;
    float* pool = nullptr;

    // Plans the sources of `count` plans; returns the pool floats they need.
    size_t plan(const cs_plan* plans, size_t count)
    {
        map.clear();
        floats = 0;
        for (size_t j = 0; j < count; ++j)
            for (int k = 0; k < plans[j].span_count; ++k) {
                const cs_voice_span& v = plans[j].spans[k];
                if (!shareable(v))
                    continue;
                WindowSource& w = map[sourceKeyOf(v)];
                w.frames = int(std::max<long long>(w.frames, sourceFramesOf(v)));
                w.channels = v.channels;
                w.users += 1;
            }
        for (auto it = map.begin(); it != map.end();) {
            if (it->second.frames <= 0) {
                it = map.erase(it);
                continue;
            }
            it->second.offset = (long long)floats;
            floats += alignFloats(size_t(it->second.frames) * size_t(it->second.channels));
            ++it;
        }
        return floats;
    }
};

// A batch's share of the window's sources: every voice whose source the window
// pools reads it there; the sources no earlier batch rendered are this batch's
// to render, from one of its voices.
SharedPlan planWindowSources(const HostBatch& batch, WindowSources& window)
{
    SharedPlan plan;
    plan.pooled = true;
    const size_t count = batch.voices.size();
    plan.refs.assign(count, SharedRef{-1, 0, 0});
    bool any = false;
    for (size_t i = 0; i < count; ++i) {
        const cs_voice_span& v = batch.voices[i];
        if (!shareable(v))
            continue;
        const auto found = window.map.find(sourceKeyOf(v));
        if (found == window.map.end())
            continue;
        WindowSource& w = found->second;
        if (!w.rendered && !w.claimed) {
            w.claimed = true;
            SharedSource source{};
            source.offset = w.offset;
            source.voice = int(i);
            source.frames = w.frames;
            plan.runs.push_back(make_int4(int(plan.sources.size()), 0, w.frames, int(plan.tiles)));
            plan.tiles += size_t(w.frames + kSourceTile - 1) / kSourceTile;
            plan.sources.push_back(source);
            plan.claims.push_back(&w);
            if (resamples(v))
                plan.sincFloats += (long long)w.frames * w.channels;
        }
        plan.refs[i] = SharedRef{w.offset, w.frames, 0};
        any = true;
        plan.sharedVoiceFrames += v.end - v.begin;
        if (resamples(v))
            plan.sincVoiceFloats += (long long)(v.end - v.begin) * v.channels;
    }
    for (WindowSource* w : plan.claims)
        w->claimed = false;
    if (!any)
        plan.refs.clear();
    if (plan.tiles > size_t(INT32_MAX))
        throw std::runtime_error("too many shared source tiles in one batch");
    return plan;
}

SharedPlan planSharedSources(const HostBatch& batch, size_t budgetBytes, WindowSources* window = nullptr)
{
    using Key = SourceKey;
    using KeyHash = SourceKeyHash;
    if (window)
        return planWindowSources(batch, *window);
    struct Entry {
        int voice = -1, frames = 0, users = 0;
        long long total = 0;
    };
    SharedPlan plan;
    const size_t count = batch.voices.size();
    // Entries live in a deque (stable addresses); the map finds them by key.
    std::deque<Entry> entryStore;
    std::unordered_map<Key, Entry*, KeyHash> entries;
    entries.reserve(count / 4 + 16);
    std::vector<const Entry*> entryOf(count, nullptr);
    for (size_t i = 0; i < count; ++i) {
        const cs_voice_span& v = batch.voices[i];
        if (!shareable(v))
            continue;
        const long long frames = sourceFramesOf(v);
        const Key key = sourceKeyOf(v);
        auto found = entries.find(key);
        if (found == entries.end()) {
            entryStore.emplace_back();
            found = entries.emplace(key, &entryStore.back()).first;
        }
        Entry& e = *found->second;
        if (e.voice < 0)
            e.voice = int(i);
        e.frames = int(std::max<long long>(e.frames, frames));
        e.users += 1;
        e.total += frames;
        entryOf[i] = &e;
    }
    // Every source, the most voice frames saved first, within the budget; in
    // order of first use among equals (deterministic).  A source only one voice
    // plays saves no resampling, but once every unfiltered voice reads a shared
    // source the mix runs without its inline resampler.
    std::vector<Entry*> chosen;
    for (Entry& e : entryStore)
        if (e.frames > 0)
            chosen.push_back(&e);
    std::stable_sort(chosen.begin(), chosen.end(), [](const Entry* a, const Entry* b) {
        return a->total - a->frames > b->total - b->frames;
    });
    std::unordered_map<const Entry*, long long> offsetOf;
    size_t bytes = 0;
    for (Entry* e : chosen) {
        const int channels = batch.voices[size_t(e->voice)].channels;
        const size_t floats = alignFloats(size_t(e->frames) * size_t(channels));
        if ((plan.floats + floats) * sizeof(float) > budgetBytes)
            continue;
        offsetOf[e] = (long long)plan.floats;
        SharedSource source{};
        source.offset = (long long)plan.floats;
        source.voice = e->voice;
        source.frames = e->frames;
        plan.runs.push_back(make_int4(int(plan.sources.size()), 0, e->frames, int(plan.tiles)));
        plan.tiles += size_t(e->frames + kSourceTile - 1) / kSourceTile;
        plan.sources.push_back(source);
        plan.floats += floats;
        if (resamples(batch.voices[size_t(e->voice)]))
            plan.sincFloats += (long long)e->frames * channels;
        bytes += floats * sizeof(float);
    }
    if (plan.sources.empty())
        return plan;
    if (plan.tiles > size_t(INT32_MAX))
        throw std::runtime_error("too many shared source tiles in one batch");
    plan.refs.assign(count, SharedRef{-1, 0, 0});
    for (size_t i = 0; i < count; ++i) {
        if (!entryOf[i])
            continue;
        const auto at = offsetOf.find(entryOf[i]);
        if (at == offsetOf.end())
            continue;
        plan.refs[i] = SharedRef{at->second, entryOf[i]->frames, 0};
        const cs_voice_span& v = batch.voices[i];
        plan.sharedVoiceFrames += v.end - v.begin;
        if (resamples(v))
            plan.sincVoiceFloats += (long long)(v.end - v.begin) * v.channels;
    }
    return plan;
}

} // namespace
} // namespace cs

namespace cs {
namespace {
class WindowRenderer;
}
}

struct cs_prepared {
    cs_renderer* owner = nullptr;
    bool sharedArena = false;
    int lane = 0;                       // the renderer lane whose streams run the batch
    cs::HostBatch batch;
    cs::SegmentTables tables;
    cs::SharedPlan shared;              // shared voice sources (empty: every source inline)
    const cs::SharedSource* sharedSources = nullptr;
    const cs::JobSpans* jobSpans = nullptr;       // device: the tile index inputs
    const int2* indexUnits = nullptr;
    const int2* sharedTiles = nullptr;
    void* arena = nullptr;
    size_t arenaBytes = 0;
    cs::BatchView view{};
    std::vector<cs::SegmentView> segments;
    cs::FinishView finish{};
    cs::StereoStats* stereo = nullptr;
    int* deferredBlocks = nullptr;      // the mix's lean pass defers blocks here
    size_t stateBytes = 0, resultBytes = 0, mixBytes = 0;
    bool natural = true;
    int launches = 0;
    cudaEvent_t begin = nullptr, end = nullptr;
    std::vector<cs_tail_result> results;
    bool ran = false;
    // Quality gate / group volume (null views when both are off).
    bool assess = false;
    bool deferGroups = false;           // a chunk of a volume group split across batches
    cs::AssessView assessView{};
    cs::PackView packView{};
    std::vector<int2> groups;           // volume groups inside the batch, job ranges
    const int2* deviceGroups = nullptr;
    size_t bodyBytes = 0;
    short* output = nullptr;            // the PCM the batch publishes
    // Download enqueued behind the batch's kernels into its lane's page-locked
    // buffer (error flag, results, PCM up to the batch's frames), done at `copied`.
    bool asyncDownload = false;
    cudaEvent_t copied = nullptr;
    cudaEvent_t downloading = nullptr;  // recorded before the download copies
    size_t downloadResults = 0, downloadPcm = 0;   // offsets in the lane's buffer
    // Optional per-stage timing: an event after every stage of the last run.
    bool profile = false;
    std::vector<cudaEvent_t> marks;
    std::vector<int> markStage;
};

struct cs_renderer {
    int device = 0;
    bool natural = true;
    cs_audio_config audio{};
    int groupMinimum = 0;
    size_t waitingLimit = 0, batchJobs = 64;
    cs::TailConfig tail{};
    std::string name;
    cudaStream_t stream = nullptr;      // lane 0's stream
    // A lane holds one batch in flight: its stream, a high-priority stream per lead
    // tier for that tier's recurrences, and the arena its batches reuse.
    struct Lane {
        cudaStream_t stream = nullptr, lead[cs::kLeadTiers] = {};
        cudaEvent_t leadReady[cs::kLeadTiers] = {}, leadDone[cs::kLeadTiers] = {};
        void* arena = nullptr;
        size_t arenaCapacity = 0;
        void* download = nullptr;       // page-locked: the lane's published batch
        size_t downloadCapacity = 0;
        void* staging = nullptr;        // page-locked: the lane's batch uploads
        size_t stagingCapacity = 0;
        cudaEvent_t uploaded = nullptr; // the lane's last uploads have been read
        cudaEvent_t staged = nullptr;   // render windows: the batch's uploads are done
        cudaEvent_t computed = nullptr; // render windows: the batch's kernels are done
    };
    static constexpr int kLanes = 4;
    Lane lanes[kLanes];
    // Render windows and serving run every lane's kernels on this one stream, in
    // batch order, while each lane's uploads and downloads stay on its own stream:
    // the oldest batch finishes first and its download starts while the next
    // batches compute (lanes computing side by side all finished late, leaving
    // the copy engines idle).
    cudaStream_t compute = nullptr;
    // Off: each lane runs its kernels on its own stream beside the others (for
    // batches whose latency-bound kernels leave the GPU room), and render windows
    // plan their shared sources per batch (nothing orders the lanes' kernels).
    bool orderedCompute = true;
    int laneCount = 2;                  // batches in flight at most (cs_renderer_set_lanes)
    float* sinc = nullptr;
    float* bank = nullptr;
    size_t bankCapacity = 0, uploaded = 0;
    size_t scratchLimit = 0;            // 0: derive from free memory
    bool sharedSources = true;          // render each shared voice source once per batch
    // Derived scratch budget (0: read it again).  cudaMemGetInfo can take
    // milliseconds while other work runs, so it is read once and kept until the
    // bank is uploaded or a batch arena does not fit.
    size_t budgetCache = 0;
    size_t deferred = 0;                // serving: launches deferred for lack of free memory
    // Largest staging, download and arena sizes any lane has needed (lanes grow to them).
    size_t stagingHigh = 0, downloadHigh = 0, arenaHigh = 0;
    size_t oomBudget = 0;               // scratch cap after a lone job's arena did not fit (0: none)
    int failAllocations = 0;            // host-side fault injection: batch arenas to refuse
    struct FailedRequest {              // sizes of the last batch whose arena did not fit
        size_t requested = 0, mix = 0, scratch = 0, finishing = 0, metadata = 0;
    } failed;
    std::string error;                  // message of this renderer's last failed call
    // Host time spent staging batches, per phase (cs_renderer_host_ms).
    double hostMs[cs::kHostPhases] = {};
    size_t peak = 0, waiting = 0, peakWaiting = 0, spilled = 0, downloaded = 0, cacheBudget = 0;
    size_t live = 0;                    // bytes of prepared batches alive
    void* hostPcm = nullptr;
    size_t hostPcmCapacity = 0;
    void* staging = nullptr;            // pinned upload buffer for batch metadata
    size_t stagingCapacity = 0;
    std::unique_ptr<cs::WorkerPool> copier;   // host copies into the staging buffer
    // The job queue and batches in flight behind cs_submit / cs_poll.
    std::unique_ptr<cs::WindowRenderer> service;
    // The shared-source pool of the render window in progress (null: batches
    // plan their own shared sources).
    cs::WindowSources* window = nullptr;
    void* windowPool = nullptr;
    size_t windowPoolCapacity = 0;

    cs::WorkerPool& copies()
    {
        if (!copier) {
            const unsigned cores = std::max(1u, std::thread::hardware_concurrency());
            copier = std::make_unique<cs::WorkerPool>(std::min(cores, 16u) - 1);
        }
        return *copier;
    }

    // Page-locked host memory that grows on demand (the copy engines read and write
    // it directly).
    // A page-locked buffer of at least `bytes`, grown with a quarter of headroom
    // and to at least `floor` (the largest size any lane has needed, so that lanes
    // taking turns at the largest batches do not each reallocate: pinning and
    // unpinning hundreds of MB stalls the host for tens of milliseconds).
    static void* pinned(void*& buffer, size_t& capacity, size_t bytes, size_t floor = 0)
    {
        if (bytes <= capacity && buffer)
            return buffer;
        if (buffer)
            cudaFreeHost(buffer);
        buffer = nullptr;
        capacity = 0;
        const size_t want = std::max<size_t>(std::max(bytes, floor) + std::max(bytes, floor) / 4, size_t(1) << 20);
        if (cudaMallocHost(&buffer, want) != cudaSuccess) {
            cudaGetLastError();
            throw std::runtime_error("cannot allocate pinned host memory");
        }
        capacity = want;
        return buffer;
    }

    void record(size_t extra = 0)
    {
        const size_t sincBytes = size_t(cs::kTaps) * (cs::kPhases + 1) * sizeof(float);
        peak = std::max(peak, sincBytes + bankCapacity * sizeof(float) + live + extra);
    }
};

namespace cs {
namespace {

using HostClock = std::chrono::steady_clock;

double msSince(HostClock::time_point& mark)
{
    const auto now = HostClock::now();
    const double ms = std::chrono::duration<double, std::milli>(now - mark).count();
    mark = now;
    return ms;
}

size_t defaultScratchBudget()
{
    size_t freeBytes = 0, total = 0;
    check(cudaMemGetInfo(&freeBytes, &total), "CUDA free memory");
    // The reference bounds a batch by min(3/4 available, total / 4); its chain
    // storage shares that budget with the mix and finishing buffers.
    return std::max<size_t>(size_t(1) << 20, std::min(freeBytes / 2, total / 4));
}

// True for page-locked host memory (cudaHostAlloc'd or registered), which the copy
// engines read directly.
bool pageLocked(const void* pointer)
{
    cudaPointerAttributes attributes{};
    if (cudaPointerGetAttributes(&attributes, pointer) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return attributes.type == cudaMemoryTypeHost;
}

// `shared`: carve the batch from the renderer's reusable arena (render_window
// batches, one alive at a time) instead of a dedicated allocation.
cs_prepared* prepare(cs_renderer& r, const cs_plan* plans, size_t count, bool shared = false, int laneIndex = 0,
                     size_t firstJob = 0)
{
    check(cudaSetDevice(r.device), "CUDA device");
    auto p = std::make_unique<cs_prepared>();
    p->owner = &r;
    p->lane = laneIndex;
    cs_renderer::Lane& lane = r.lanes[laneIndex];
    p->natural = r.natural;
    HostBatch& batch = p->batch;
    const bool assess = r.audio.enabled || r.groupMinimum > 0;
    const BodyGeometry body = bodyGeometry(r.audio);
    auto mark = HostClock::now();
    batch.build(plans, count, r.tail.window, r.natural, assess, r.audio.enabled != 0, body, r.copies());
    r.hostMs[0] += msSince(mark);
    p->assess = assess;
    if (assess && r.groupMinimum > 0) {
        // Volume groups: runs of equal nonzero ids (src/cuda/renderer.cpp:1751-1761).
        const auto& ids = batch.volumeGroups;
        for (size_t first = 0, end; first < ids.size(); first = end) {
            end = first + 1;
            if (!ids[first])
                continue;
            while (end < ids.size() && ids[end] == ids[first])
                ++end;
            p->groups.push_back(make_int2(int(first), int(end)));
        }
    }
    // The derived budget is read once and kept (cudaMemGetInfo is slow).
    if (!r.scratchLimit && !r.budgetCache)
        r.budgetCache = defaultScratchBudget();
    size_t scratchBudget = r.scratchLimit ? r.scratchLimit : r.budgetCache;
    if (r.oomBudget)
        scratchBudget = std::min(scratchBudget, r.oomBudget);
    r.hostMs[1] += msSince(mark);
    p->tables = planSegments(batch, scratchBudget);
    const SegmentTables& t = p->tables;
    if (t.segments.size() > 1)          // the reference's protocol line for segmented synthesis
        std::fprintf(stderr, "SEGMENT\tfirst=%zu\tjobs=%zu\tcount=%zu\tscratch_bytes=%zu\tfull_scratch_bytes=%zu\n",
                     firstJob, count, t.segments.size(), t.scratchBytes, t.fullScratchBytes);
    r.hostMs[2] += msSince(mark);
    if (r.sharedSources)
        p->shared = planSharedSources(batch, scratchBudget / 2, r.window);
    r.hostMs[3] += msSince(mark);
    const SharedPlan& sh = p->shared;
    const size_t jobs = batch.jobs.size();
    const size_t frameBytes = r.natural ? sizeof(float2) : sizeof(short2);
    const int channels = r.natural ? 1 : 2;

    Layout layout;
    const auto section = [&](size_t bytes) { return layout.add(std::max<size_t>(bytes, 1)); };
    const size_t oVoices = section(batch.voices.size() * sizeof(cs_voice_span));
    const size_t oPoints = section(batch.pointCount * sizeof(cs_control_point));
    const size_t oMods = section(batch.modulation.size() * sizeof(cs_voice_modulation));
    const size_t oJobs = section(jobs * sizeof(JobInfo));
    const size_t oJobSpans = section(batch.jobSpans.size() * sizeof(JobSpans));
    const size_t oIndexUnits = section(batch.indexUnits.size() * sizeof(int2));
    const size_t oBlockJob = section(batch.blockJob.size() * sizeof(int));
    const size_t oWindowJob = section(batch.windowJob.size() * sizeof(int));
    const size_t oScratchOff = section(t.scratchOffset.size() * sizeof(uint64_t));
    const size_t oPhaseOff = section(t.phaseOffset.size() * sizeof(uint64_t));
    const size_t oTargetOff = section(t.targetOffset.size() * sizeof(uint64_t));
    const size_t oTileRuns = section(t.tileRuns.size() * sizeof(int4));
    const size_t oChains = section(t.chains.size() * sizeof(int));
    const size_t oSimple = section(t.simple.size() * sizeof(int));
    const size_t oPitch = section(t.pitch.size() * sizeof(int));
    const size_t oBlocks = section(t.blocks.size() * sizeof(int));
    const size_t oJobBlockFirst = section(batch.jobBlockFirst.size() * sizeof(int));
    const size_t oAssess = section(batch.assess.size() * sizeof(AssessJob));
    const size_t oOnsets = section(batch.onsets.size() * sizeof(int));
    const size_t oOnsetJob = section(batch.onsetJob.size() * sizeof(int));
    const size_t oGroups = section(p->groups.size() * sizeof(int2));
    const size_t oSharedSources = section(sh.sources.size() * sizeof(SharedSource));
    const size_t oSharedRefs = section(sh.refs.size() * sizeof(SharedRef));
    const size_t oSharedRuns = section(sh.runs.size() * sizeof(int4));
    const size_t uploadEnd = layout.bytes;
    p->stateBytes = batch.voices.size() * sizeof(ChainState);
    const size_t oStates = section(p->stateBytes);
    const size_t oTiles = section(batch.tileCount * sizeof(MixTile));
    const size_t oIndices = section(batch.indexCount * sizeof(int));
    p->resultBytes = jobs * sizeof(cs_tail_result);
    const size_t oResults = section(p->resultBytes);
    const size_t oScans = section(jobs * sizeof(JobScan));
    p->mixBytes = batch.frames * frameBytes;
    const size_t oMix = section(p->mixBytes);
    const size_t oStereo = section(size_t(batch.blocks) * sizeof(StereoStats));
    const size_t oDeferred = section((size_t(batch.blocks) + 1) * sizeof(int));
    const size_t oWindows = section(size_t(batch.windows) * sizeof(MonoStats));
    const size_t oMono = section(r.natural ? batch.frames * sizeof(short) : 0);
    const size_t oPacked = section(batch.frames * size_t(channels) * sizeof(short));
    const size_t oSourceTiles = section(t.tileCount * sizeof(int2));
    const size_t oSharedTiles = section(sh.tiles * sizeof(int2));
    const size_t oShared = section(sh.pooled ? 0 : sh.floats * sizeof(float));
    const size_t oScratch = section(t.scratchBytes);
    const size_t oError = section(sizeof(int));
    p->bodyBytes = size_t(batch.bodyWindows) * sizeof(unsigned long long);
    const size_t oBodyPower = section(p->bodyBytes);
    const size_t oOnsetPower = section(batch.onsets.size() * sizeof(unsigned long long));
    const size_t oSourceOffset = section(assess ? jobs * sizeof(uint64_t) : 0);
    p->arenaBytes = layout.bytes;

    if (shared) {
        if (p->arenaBytes > lane.arenaCapacity) {
            cudaFree(lane.arena);
            r.live -= lane.arenaCapacity;
            lane.arena = nullptr;
            lane.arenaCapacity = 0;
            // Grown to the largest arena any lane has needed, with an eighth of
            // headroom, falling back to the exact size when that does not fit.
            r.arenaHigh = std::max(r.arenaHigh, p->arenaBytes);
            size_t want = r.arenaHigh + r.arenaHigh / 8;
            cudaError_t status = r.failAllocations > 0 ? cudaErrorMemoryAllocation : cudaMalloc(&lane.arena, want);
            if (status == cudaErrorMemoryAllocation && r.failAllocations <= 0 && want > p->arenaBytes) {
                cudaGetLastError();
                want = p->arenaBytes;
                status = cudaMalloc(&lane.arena, want);
            }
            if (r.failAllocations > 0)
                --r.failAllocations;
            if (status != cudaSuccess) {
                cudaGetLastError();
                lane.arena = nullptr;
                r.failed = {p->arenaBytes, p->mixBytes, t.scratchBytes, oScratch - oMix - p->mixBytes,
                            uploadEnd};
                throw CudaError(status, "CUDA batch arena allocation");
            }
            lane.arenaCapacity = want;
            r.live += lane.arenaCapacity;
        }
        p->arena = lane.arena;
        p->sharedArena = true;
    } else {
        cudaError_t status = r.failAllocations > 0 ? cudaErrorMemoryAllocation : cudaMalloc(&p->arena, p->arenaBytes);
        if (r.failAllocations > 0)
            --r.failAllocations;
        if (status != cudaSuccess) {
            cudaGetLastError();
            p->arena = nullptr;
            r.failed = {p->arenaBytes, p->mixBytes, t.scratchBytes, oScratch - oMix - p->mixBytes, uploadEnd};
            throw CudaError(status, "CUDA batch arena allocation");
        }
        r.live += p->arenaBytes;
    }
    r.record();
    r.hostMs[4] += msSince(mark);
    auto* base = static_cast<unsigned char*>(p->arena);
    // Render-window batches stage through their lane's buffer, reused once the
    // lane's previous uploads have been read; other batches use the renderer's.
    if (shared && lane.uploaded)
        check(cudaEventSynchronize(lane.uploaded), "CUDA staging reuse");
    if (shared)
        r.stagingHigh = std::max(r.stagingHigh, uploadEnd);
    auto* staging = static_cast<unsigned char*>(
        shared ? cs_renderer::pinned(lane.staging, lane.stagingCapacity, uploadEnd, r.stagingHigh)
               : cs_renderer::pinned(r.staging, r.stagingCapacity, uploadEnd));
    std::vector<CopyPiece> pieces;
    const auto stage = [&](size_t offset, const auto& items) {
        if (!items.empty())
            pieces.push_back({staging + offset, items.data(), items.size() * sizeof(items.front())});
    };
    stage(oVoices, batch.voices);
    // Control points already in page-locked memory go to the device straight from
    // the caller's arrays; the rest pass through the staging buffer.
    std::vector<CopyPiece> direct;
    {
        size_t at = oPoints;
        for (const auto& [first, count] : batch.pointSources) {
            const size_t bytes = count * sizeof(cs_control_point);
            if (!bytes)
                continue;
            // Large page-locked arrays go up directly; small ones are cheaper to copy
            // into the staging buffer than to upload one by one.
            if (bytes >= (size_t(256) << 10) && pageLocked(first))
                direct.push_back({base + at, first, bytes});
            else
                pieces.push_back({staging + at, first, bytes});
            at += bytes;
        }
    }
    stage(oMods, batch.modulation);
    stage(oJobs, batch.jobs);
    stage(oJobSpans, batch.jobSpans);
    stage(oIndexUnits, batch.indexUnits);
    stage(oBlockJob, batch.blockJob);
    stage(oWindowJob, batch.windowJob);
    stage(oScratchOff, t.scratchOffset);
    stage(oPhaseOff, t.phaseOffset);
    stage(oTargetOff, t.targetOffset);
    stage(oTileRuns, t.tileRuns);
    stage(oChains, t.chains);
    stage(oSimple, t.simple);
    stage(oPitch, t.pitch);
    stage(oBlocks, t.blocks);
    stage(oJobBlockFirst, batch.jobBlockFirst);
    stage(oAssess, batch.assess);
    stage(oOnsets, batch.onsets);
    stage(oOnsetJob, batch.onsetJob);
    stage(oGroups, p->groups);
    stage(oSharedSources, sh.sources);
    stage(oSharedRefs, sh.refs);
    stage(oSharedRuns, sh.runs);
    // Copy and upload the staged ranges in slices: each slice's DMA runs while the
    // workers copy the next slice.  Ranges are the staged pieces merged across small
    // gaps (section alignment); the direct uploads follow them in stream order, so
    // a merged range never leaves stale bytes over a directly uploaded piece.
    r.hostMs[5] += msSince(mark);
    std::vector<std::pair<size_t, size_t>> ranges;
    for (const CopyPiece& piece : pieces) {
        const size_t a = size_t(static_cast<unsigned char*>(piece.dst) - staging), b = a + piece.bytes;
        if (!ranges.empty() && a <= ranges.back().second + 4096)
            ranges.back().second = std::max(ranges.back().second, b);
        else
            ranges.emplace_back(a, b);
    }
    constexpr size_t kSlice = size_t(128) << 20;
    for (const auto& [rangeFirst, rangeEnd] : ranges) {
        for (size_t from = rangeFirst; from < rangeEnd; from += kSlice) {
            const size_t to = std::min(rangeEnd, from + kSlice);
            std::vector<CopyPiece> slice;
            for (const CopyPiece& piece : pieces) {
                const size_t a = size_t(static_cast<unsigned char*>(piece.dst) - staging), b = a + piece.bytes;
                const size_t lo = std::max(a, from), hi = std::min(b, to);
                if (lo < hi)
                    slice.push_back({staging + lo, static_cast<const unsigned char*>(piece.src) + (lo - a), hi - lo});
            }
            r.copies().copy(slice);
            check(cudaMemcpyAsync(base + from, staging + from, to - from, cudaMemcpyHostToDevice, lane.stream),
                  "CUDA batch upload");
        }
    }
    for (const CopyPiece& piece : direct)
        check(cudaMemcpyAsync(piece.dst, piece.src, piece.bytes, cudaMemcpyHostToDevice, lane.stream),
              "CUDA batch upload");
    // The source tiles (256 frames of one span each) are expanded from the runs on
    // the device: millions of them for an hour of voices.
    launchExpandTiles(reinterpret_cast<const int4*>(base + oTileRuns), int(t.tileRuns.size()),
                      reinterpret_cast<int2*>(base + oSourceTiles), lane.stream);
    launchExpandTiles(reinterpret_cast<const int4*>(base + oSharedRuns), int(sh.runs.size()),
                      reinterpret_cast<int2*>(base + oSharedTiles), lane.stream);
    check(cudaGetLastError(), "CUDA source tile expansion");
    r.hostMs[6] += msSince(mark);
    if (shared) {
        // The batch runs on the lane's stream after its uploads; the staging buffer
        // is reused once this event has passed.
        if (!lane.uploaded)
            check(cudaEventCreateWithFlags(&lane.uploaded, cudaEventDisableTiming), "CUDA upload event");
        check(cudaEventRecord(lane.uploaded, lane.stream), "CUDA upload event");
    } else {
        check(cudaStreamSynchronize(lane.stream), "CUDA batch upload");
    }
    r.hostMs[7] += msSince(mark);

    BatchView& v = p->view;
    v.bank = r.bank;
    v.sinc = r.sinc;
    v.voices = reinterpret_cast<const cs_voice_span*>(base + oVoices);
    v.points = reinterpret_cast<const cs_control_point*>(base + oPoints);
    v.modulation = reinterpret_cast<const cs_voice_modulation*>(base + oMods);
    v.jobs = reinterpret_cast<const JobInfo*>(base + oJobs);
    v.tiles = reinterpret_cast<const MixTile*>(base + oTiles);
    v.indices = reinterpret_cast<const int*>(base + oIndices);
    v.blockJob = reinterpret_cast<const int*>(base + oBlockJob);
    v.windowJob = reinterpret_cast<const int*>(base + oWindowJob);
    v.states = reinterpret_cast<ChainState*>(base + oStates);
    p->jobSpans = reinterpret_cast<const JobSpans*>(base + oJobSpans);
    p->indexUnits = reinterpret_cast<const int2*>(base + oIndexUnits);
    v.filtered = reinterpret_cast<float*>(base + oScratch);
    v.mix = base + oMix;
    v.error = reinterpret_cast<int*>(base + oError);
    v.shared = sh.pooled ? r.window->pool : reinterpret_cast<float*>(base + oShared);
    v.sharedRefs = sh.refs.empty() ? nullptr : reinterpret_cast<const SharedRef*>(base + oSharedRefs);
    p->sharedSources = reinterpret_cast<const SharedSource*>(base + oSharedSources);
    p->sharedTiles = reinterpret_cast<const int2*>(base + oSharedTiles);
    v.jobCount = int(jobs);
    // 1: the mix resamples some unfiltered voice itself; 2: every unfiltered voice
    // reads a shared source; 0: no unfiltered voice.
    v.inlineVoices = 0;
    for (size_t k = 0; k < batch.voices.size(); ++k) {
        if (batch.voices[k].filterTrack >= 0)
            continue;
        if (sh.refs.empty() || sh.refs[k].offset < 0) {
            v.inlineVoices = 1;
            break;
        }
        v.inlineVoices = 2;
    }
    const size_t voiceCount = batch.voices.size();
    for (const auto& seg : t.segments) {
        SegmentView s{};
        const size_t si = size_t(&seg - t.segments.data());
        s.first = seg.first;
        s.end = seg.end;
        s.scratchOffset = reinterpret_cast<const uint64_t*>(base + oScratchOff) + si * voiceCount;
        s.phaseOffset = reinterpret_cast<const uint64_t*>(base + oPhaseOff) + si * voiceCount;
        s.chains = reinterpret_cast<const int*>(base + oChains) + seg.chainFirst;
        s.chainCount = int(seg.chainCount);
        s.simple = reinterpret_cast<const int*>(base + oSimple) + seg.simpleFirst;
        s.simpleCount = int(seg.simpleCount);
        s.targetOffset = reinterpret_cast<const uint64_t*>(base + oTargetOff) + si * voiceCount;
        s.sourceTiles = reinterpret_cast<const int2*>(base + oSourceTiles) + seg.tileFirst;
        s.sourceTileCount = int(seg.tileCount);
        s.pitchChains = reinterpret_cast<const int*>(base + oPitch) + seg.pitchFirst;
        s.pitchCount = int(seg.pitchCount);
        s.blocks = reinterpret_cast<const int*>(base + oBlocks) + seg.blockFirst;
        s.blockCount = int(seg.blockCount);
        p->segments.push_back(s);
    }
    // Pitch phases follow the filtered floats of the same segment.
    v.phase = reinterpret_cast<double*>(base + oScratch);
    FinishView& f = p->finish;
    f.scans = reinterpret_cast<JobScan*>(base + oScans);
    f.stereo = reinterpret_cast<StereoStats*>(base + oStereo);
    f.windows = reinterpret_cast<MonoStats*>(base + oWindows);
    f.mono = reinterpret_cast<short*>(base + oMono);
    f.packed = reinterpret_cast<short*>(base + oPacked);
    f.results = reinterpret_cast<cs_tail_result*>(base + oResults);
    f.blockCount = batch.blocks;
    f.windowCount = batch.windows;
    p->stereo = f.stereo;
    p->deferredBlocks = reinterpret_cast<int*>(base + oDeferred);
    p->output = f.packed;
    if (assess) {
        f.bodyPower = reinterpret_cast<unsigned long long*>(base + oBodyPower);
        f.assess = reinterpret_cast<const AssessJob*>(base + oAssess);
        f.body = body;
        AssessView& a = p->assessView;
        a.jobs = f.assess;
        a.onsets = reinterpret_cast<const int*>(base + oOnsets);
        a.onsetJob = reinterpret_cast<const int*>(base + oOnsetJob);
        a.bodyPower = f.bodyPower;
        a.onsetPower = reinterpret_cast<unsigned long long*>(base + oOnsetPower);
        a.config = r.audio;
        a.body = body;
        a.jobCount = int(jobs);
        a.onsetCount = int(batch.onsets.size());
        p->deviceGroups = reinterpret_cast<const int2*>(base + oGroups);
        // Accepted PCM goes to a buffer that is dead once finishing is done: the
        // mono quantisation (natural) or the PCM16 mix (orig/custom).
        p->output = r.natural ? f.mono : static_cast<short*>(v.mix);
        PackView& k = p->packView;
        k.blockJob = v.blockJob;
        k.jobBlockFirst = reinterpret_cast<const int*>(base + oJobBlockFirst);
        k.results = f.results;
        k.sourceOffset = reinterpret_cast<uint64_t*>(base + oSourceOffset);
        k.source = f.packed;
        k.output = p->output;
        k.jobCount = int(jobs);
        k.blockCount = batch.blocks;
    }
    check(cudaEventCreate(&p->begin), "CUDA timing event");
    check(cudaEventCreate(&p->end), "CUDA timing event");
    return p.release();
}

const char* const kStageNames[] = {"pitch", "source", "recurrence", "general", "mix", "finish", "assess", "shared",
                                   "index"};
constexpr int kStages = 9;

void run(cs_renderer& r, cs_prepared& p, cudaStream_t stream)
{
    check(cudaSetDevice(r.device), "CUDA device");
    if (!stream)
        stream = r.lanes[p.lane].stream;
    p.view.bank = r.bank;
    p.view.sinc = r.sinc;
    int launches = 0;
    size_t mark = 0;
    p.markStage.clear();
    const auto stage = [&](int id) {
        if (!p.profile)
            return;
        if (mark == p.marks.size()) {
            cudaEvent_t e;
            check(cudaEventCreate(&e), "CUDA timing event");
            p.marks.push_back(e);
        }
        check(cudaEventRecord(p.marks[mark++], stream), "CUDA timing record");
        p.markStage.push_back(id);
    };
    check(cudaEventRecord(p.begin, stream), "CUDA timing record");
    check(cudaMemsetAsync(p.view.states, 0, std::max<size_t>(p.stateBytes, 1), stream), "CUDA state reset");
    check(cudaMemsetAsync(p.finish.results, 0, std::max<size_t>(p.resultBytes, 1), stream), "CUDA result reset");
    check(cudaMemsetAsync(p.view.error, 0, sizeof(int), stream), "CUDA error flag reset");
    if (p.bodyBytes)
        check(cudaMemsetAsync(p.finish.bodyPower, 0, p.bodyBytes, stream), "CUDA body power reset");
    stage(-1);
    launchTileIndex(p.view, p.jobSpans, p.indexUnits, int(p.batch.indexUnits.size()), const_cast<MixTile*>(p.view.tiles),
                    const_cast<int*>(p.view.indices), stream);
    launches += p.batch.indexUnits.empty() ? 0 : 1;
    stage(8);
    launches += launchSharedSources(p.view, p.sharedSources, p.sharedTiles, int(p.shared.tiles), stream);
    stage(7);
    for (size_t i = 0; i < p.segments.size(); ++i) {
        BatchView view = p.view;
        const SegmentPlan& plan = p.tables.segments[i];
        view.phase = reinterpret_cast<double*>(reinterpret_cast<unsigned char*>(view.filtered) +
                                               align256(plan.scratchFloats * sizeof(float)));
        const SegmentView& s = p.segments[i];
        launchPitch(view, s, stream);
        launches += s.pitchCount > 0;
        stage(0);
        if (plan.leadTiers) {
            // Each lead tier's sources, then its recurrences on that tier's
            // high-priority stream beside the later tiers' and the rest's sources;
            // the rest's recurrences last, then the join.
            const cs_renderer::Lane& lane = r.lanes[p.lane];
            SegmentView rest = s;
            for (int k = 0; k < plan.leadTiers; ++k) {
                SegmentView tier = rest;
                tier.sourceTileCount = int(plan.leadTiles[k]);
                tier.simpleCount = int(plan.leadChains[k]);
                rest.sourceTiles += plan.leadTiles[k];
                rest.sourceTileCount -= int(plan.leadTiles[k]);
                rest.simple += plan.leadChains[k];
                rest.simpleCount -= int(plan.leadChains[k]);
                launches += launchSources(view, tier, stream);
                check(cudaEventRecord(lane.leadReady[k], stream), "CUDA event record");
                check(cudaStreamWaitEvent(lane.lead[k], lane.leadReady[k], 0), "CUDA stream wait");
                launches += launchRecurrences(view, tier, lane.lead[k]);
                check(cudaEventRecord(lane.leadDone[k], lane.lead[k]), "CUDA event record");
            }
            launches += launchSources(view, rest, stream);
            stage(1);
            launches += launchRecurrences(view, rest, stream);
            for (int k = 0; k < plan.leadTiers; ++k)
                check(cudaStreamWaitEvent(stream, lane.leadDone[k], 0), "CUDA stream wait");
        } else {
            launches += launchSources(view, s, stream);
            stage(1);
            launches += launchRecurrences(view, s, stream);
        }
        stage(2);
        launches += launchGeneralChains(view, s, stream);
        stage(3);
        launches += launchMix(view, s, r.natural, p.stereo, p.deferredBlocks, stream);
        stage(4);
    }
    check(cudaGetLastError(), "CUDA synthesis launch");
    launches += launchFinish(p.view, p.finish, r.natural, r.audio.enabled != 0, r.tail, stream);
    stage(5);
    check(cudaGetLastError(), "CUDA finishing launch");
    if (p.assess) {
        // Quality gate and group volume (src/cuda/renderer.cpp:1170-1180, 1134-1148):
        // verdicts, then the gains of the groups the batch holds whole, then the
        // accepted PCM.  A chunk of a split group stops after the verdicts; its
        // caller matches the whole group and packs each chunk.
        launches += launchMeasure(p.assessView, p.finish.results, p.finish.packed, r.natural, stream);
        if (!p.deferGroups) {
            if (r.groupMinimum > 0)
                launches += launchMatch(p.deviceGroups, int(p.groups.size()), r.groupMinimum, p.finish.results, stream);
            launches += launchPack(p.packView, r.natural, stream);
        }
        stage(6);
        check(cudaGetLastError(), "CUDA assessment launch");
    }
    check(cudaEventRecord(p.end, stream), "CUDA timing record");
    p.launches = launches;
    p.ran = true;
}

// Synchronises and reads the results; returns the packed PCM sample count.
size_t collectResults(cs_renderer& r, cs_prepared& p)
{
    check(cudaEventSynchronize(p.end), "CUDA render completion");
    int failed = 0;
    check(cudaMemcpy(&failed, p.view.error, sizeof(int), cudaMemcpyDeviceToHost), "CUDA error flag download");
    if (failed)
        throw std::runtime_error("a device wait ran out of its iteration limit (staged copy did not complete)");
    p.results.resize(p.batch.jobs.size());
    check(cudaMemcpy(p.results.data(), p.finish.results, p.resultBytes, cudaMemcpyDeviceToHost),
          "CUDA render metadata download");
    if (p.results.empty())
        return 0;
    const auto& last = p.results.back();
    return size_t(last.offset + uint64_t(last.dataFrames)) * (r.natural ? 1 : 2);
}

// Enqueues the batch's download behind its kernels on its lane's stream: the error
// flag, the results and the PCM (up to the batch's frames, an upper bound of what
// it publishes) into the lane's page-locked buffer, so that the copy runs while
// the host stages the next batch.  The lane's previous batch is already published.
void enqueueDownload(cs_renderer& r, cs_prepared& p)
{
    cs_renderer::Lane& lane = r.lanes[p.lane];
    const size_t pcmBytes = p.batch.frames * (r.natural ? 1 : 2) * sizeof(int16_t);
    p.downloadResults = 256;
    p.downloadPcm = align256(p.downloadResults + p.resultBytes);
    auto* buffer = static_cast<unsigned char*>(
        cs_renderer::pinned(lane.download, lane.downloadCapacity, p.downloadPcm + std::max<size_t>(pcmBytes, 1),
                            r.downloadHigh = std::max(r.downloadHigh, p.downloadPcm + std::max<size_t>(pcmBytes, 1))));
    if (!p.copied)
        check(cudaEventCreate(&p.copied), "CUDA download event");
    if (!p.downloading)
        check(cudaEventCreate(&p.downloading), "CUDA download event");
    check(cudaEventRecord(p.downloading, lane.stream), "CUDA download event");
    check(cudaMemcpyAsync(buffer, p.view.error, sizeof(int), cudaMemcpyDeviceToHost, lane.stream), "CUDA error flag download");
    check(cudaMemcpyAsync(buffer + p.downloadResults, p.finish.results, p.resultBytes, cudaMemcpyDeviceToHost, lane.stream),
          "CUDA render metadata download");
    if (pcmBytes)
        check(cudaMemcpyAsync(buffer + p.downloadPcm, p.output, pcmBytes, cudaMemcpyDeviceToHost, lane.stream),
              "CUDA PCM download");
    check(cudaEventRecord(p.copied, lane.stream), "CUDA download event");
    p.asyncDownload = true;
}

void checkPlans(const cs_plan* plans, size_t count)
{
    if (count && !plans)
        throw std::runtime_error("null plan array");
    for (size_t i = 0; i < count; ++i) {
        const cs_plan& p = plans[i];
        if (p.frames <= 0 || (p.span_count && !p.spans) || p.track_count < 3 || !p.track_offsets ||
            (p.modulation_count && !p.modulation))
            throw std::runtime_error("invalid plan " + std::to_string(i));
    }
}

template <class F>
int guarded(F&& body)
{
    try {
        body();
        return 0;
    } catch (const std::exception& e) {
        lastError = e.what();
        return 1;
    }
}

// As guarded, and the message is also kept on the renderer (cs_renderer_last_error).
template <class F>
int guardedOn(cs_renderer* r, F&& body);


// Renderer::renderWindow (src/cuda/renderer.cpp:1748-1820) over staged batches.
// Batches take up to batchJobs plans and never cut a volume group unless the group
// alone exceeds a batch; such a group is rendered in chunks whose accepted PCM
// waits on the device (within the waiting limit) or in host memory until the last
// chunk's verdicts are in, then every chunk is packed with the group's gains
// (finishSplit, retain and packRetained, renderer.cpp:1206-1346).
class WindowRenderer {
public:
    WindowRenderer(cs_renderer& renderer, cs_publish_fn publish, cs_refill_fn refill, void* user)
        : r(renderer), publish(publish), refill(refill), user(user) {}

    ~WindowRenderer()
    {
        for (const InFlight& f : flight)       // after an error: unpublished batches
            cs_prepared_destroy(f.batch);
    }

    void render(const cs_plan* plans, size_t count)
    {
        r.oomBudget = 0;
        queue.assign(plans, plans + count);
        next = 0;
        // One shared-source pool for the whole window (volume groups render
        // their chunks apart, so they keep per-batch sources).  A worker thread
        // plans it while the first batch is staged with sources of its own; the
        // pool serves the batches from the second on.
        WindowSources window;
        struct Detach {
            WindowRenderer& w;
            ~Detach()
            {
                if (w.windowPlan.valid())
                    w.windowPlan.wait();
                w.r.window = nullptr;
                w.pendingWindow = nullptr;
            }
        } detach{*this};
        r.window = nullptr;
        pendingWindow = nullptr;
        if (r.sharedSources && r.orderedCompute && r.groupMinimum <= 0) {
            pendingWindow = &window;
            windowPlan = std::async(std::launch::async, [&window, plans, count] { return window.plan(plans, count); });
        }
        for (;;) {
            launch(true);
            if (flight.empty())
                break;
            publishFront();
        }
        // The reference's summary line of a render window (jobs, batches, refills).
        std::fprintf(stderr, "SCHEDULE\tjobs=%zu\trounds=%zu\trefills=%zu\n", queue.size(), rounds, refills);
    }

    // The window planned on the worker thread, attached once a batch is in flight.
    WindowSources* pendingWindow = nullptr;
    std::future<size_t> windowPlan;

    void attachWindow()
    {
        if (!pendingWindow || flight.empty())
            return;
        WindowSources& window = *pendingWindow;
        pendingWindow = nullptr;
        const size_t floats = windowPlan.get();
        r.window = poolWindow(window, floats) ? &window : nullptr;
    }

    // Places the pool of a planned window (`floats` floats), within half the
    // scratch budget; false when nothing is shared or the pool does not fit.
    bool poolWindow(WindowSources& window, size_t floats)
    {
        if (!floats)
            return false;
        if (!r.scratchLimit && !r.budgetCache)
            r.budgetCache = defaultScratchBudget();
        const size_t bytes = floats * sizeof(float);
        if (bytes > (r.scratchLimit ? r.scratchLimit : r.budgetCache) / 2)
            return false;
        if (bytes > r.windowPoolCapacity) {
            cudaFree(r.windowPool);
            r.live -= r.windowPoolCapacity;
            r.windowPool = nullptr;
            r.windowPoolCapacity = 0;
            const size_t want = bytes + bytes / 8;
            if (cudaMalloc(&r.windowPool, want) != cudaSuccess) {
                cudaGetLastError();
                r.windowPool = nullptr;
                return false;
            }
            r.windowPoolCapacity = want;
            r.live += want;
            r.record();
        }
        window.pool = static_cast<float*>(r.windowPool);
        return true;
    }

    // cs_submit: queues plans and launches what the free lanes take; returns the
    // ticket (queue position) of the first plan.
    size_t submit(const cs_plan* plans, size_t count)
    {
        const size_t ticket = ticketBase + queue.size();
        r.oomBudget = 0;
        queue.insert(queue.end(), plans, plans + count);
        launch(false, true);
        return ticket;
    }

    // cs_poll: publishes the oldest batch in flight once it is done (waiting for it
    // when `wait`), then launches queued plans into the lanes that freed up.
    // Returns the jobs published.
    size_t poll(bool wait, cs_publish_fn fn, void* data)
    {
        publish = fn;
        user = data;
        size_t published = 0;
        // Every finished batch is published, in the order they finish (a short
        // job's batch does not wait for an older, longer one); with `wait`, the
        // oldest is waited for when none has finished.
        for (;;) {
            auto done = flight.end();
            for (auto f = flight.begin(); f != flight.end(); ++f) {
                const cudaError_t state = cudaEventQuery(f->batch->copied ? f->batch->copied : f->batch->end);
                if (state != cudaSuccess && state != cudaErrorNotReady)
                    check(state, "CUDA batch completion");
                if (state == cudaSuccess) {
                    done = f;
                    break;
                }
            }
            if (done == flight.end()) {
                if (!wait || flight.empty())
                    break;
                done = flight.begin();
            }
            wait = false;                       // one blocking wait per call at most
            InFlight item = *done;
            flight.erase(done);
            published += item.batch->batch.jobs.size();
            std::unique_ptr<cs_prepared, void (*)(cs_prepared*)> guard(item.batch, cs_prepared_destroy);
            publishBatch(*item.batch, item.first);
            guard.reset();
            launch(false, true);
        }
        launch(false, true);
        dropPublished();
        return published;
    }

    // Serving: forget the queued plans every batch has taken, keeping tickets
    // (queue positions) stable through a base offset.
    void dropPublished()
    {
        size_t oldest = next;
        for (const InFlight& f : flight)
            oldest = std::min(oldest, f.first);
        if (oldest < 4096 || oldest < queue.size() / 2 || !chunks.empty())
            return;
        queue.erase(queue.begin(), queue.begin() + std::ptrdiff_t(oldest));
        for (InFlight& f : flight)
            f.first -= oldest;
        next -= oldest;
        ticketBase += oldest;
    }

    size_t pending() const { return queue.size() - next; }
    size_t inFlight() const { return flight.size(); }
    size_t inFlightJobs() const
    {
        size_t jobs = 0;
        for (const InFlight& f : flight)
            jobs += f.batch->batch.jobs.size();
        return jobs;
    }

private:
    size_t next = 0;                            // first queued plan not yet launched
    size_t ticketBase = 0;                      // tickets of the plans dropped from the queue
    size_t rounds = 0, refills = 0;             // batches launched, refills taken

    // Keeps up to laneCount batches in flight: the next batch is staged and
    // launched on a free lane while the others run.  `mayRefill`: ask the refill
    // callback for more plans when the queue runs dry.  `admit`: while batches are
    // in flight, launch another only if its estimated device footprint fits in half
    // of the free device memory (the reference's admission of resident jobs,
    // src/cuda/renderer.cpp:1447-1481).
    void launch(bool mayRefill, bool admit = false)
    {
        size_t freeBytes = 0;
        bool freeKnown = false;
        while (flight.size() < size_t(std::clamp(r.laneCount, 1, cs_renderer::kLanes))) {
            if (next == queue.size() && !(mayRefill && more(flight.empty())))
                break;
            // With nothing in flight, a quarter batch starts the device and the
            // download sooner while the host stages the rest (volume groups keep
            // whole batches, so their chunking does not change).
            const size_t want = flight.empty() && r.groupMinimum <= 0 && queue.size() - next > r.batchJobs
                ? std::max<size_t>(1, r.batchJobs / 4) : r.batchJobs;
            size_t jobs = batchEnd(next, std::min(queue.size(), next + want)) - next;
            if (admit && !flight.empty()) {
                if (!freeKnown) {
                    size_t total = 0;
                    check(cudaMemGetInfo(&freeBytes, &total), "CUDA free memory");
                    freeKnown = true;
                }
                if (footprint(next, jobs) > freeBytes / 2) {
                    ++r.deferred;
                    break;
                }
            }
            if (splitGroup(next, jobs)) {
                // Chunks of a volume group larger than a batch go one at a time.
                drain();
                next = renderAlone(next, jobs);
                continue;
            }
            attachWindow();
            const int lane = freeLane();
            cs_prepared* prepared = tryPrepare(next, jobs, lane);
            if (!prepared) {
                drain();
                next = rejectJob(next);
                continue;
            }
            if (splitGroup(next, jobs)) {              // a smaller batch now cuts a group
                cs_prepared_destroy(prepared);
                drain();
                next = renderAlone(next, jobs);
                continue;
            }
            if (r.orderedCompute) {
                cs_renderer::Lane& l = r.lanes[prepared->lane];
                check(cudaEventRecord(l.staged, l.stream), "CUDA event record");
                check(cudaStreamWaitEvent(r.compute, l.staged, 0), "CUDA stream wait");
                run(r, *prepared, r.compute);
                for (WindowSource* w : prepared->shared.claims)
                    w->rendered = true;
                check(cudaEventRecord(l.computed, r.compute), "CUDA event record");
                check(cudaStreamWaitEvent(l.stream, l.computed, 0), "CUDA stream wait");
            } else {
                run(r, *prepared, nullptr);
            }
            enqueueDownload(r, *prepared);
            ++rounds;
            flight.push_back({prepared, next});
            next += jobs;
            freeKnown = false;
        }
    }

    int freeLane() const
    {
        for (int lane = 0; lane < cs_renderer::kLanes; ++lane) {
            bool busy = false;
            for (const InFlight& f : flight)
                busy |= f.batch->lane == lane;
            if (!busy)
                return lane;
        }
        return 0;
    }

    // Device bytes a batch of `jobs` queued plans needs, estimated from its frames
    // and spans: the float mix, mono and packed PCM, tail statistics and the span
    // records (the arena's large sections).
    size_t footprint(size_t first, size_t jobs) const
    {
        size_t frames = 0, spans = 0;
        for (size_t j = first; j < first + jobs; ++j) {
            frames += size_t(queue[j].frames);
            spans += size_t(queue[j].span_count);
        }
        return frames * (sizeof(float2) + 3 * sizeof(short)) + spans * (sizeof(cs_voice_span) + sizeof(ChainState));
    }

private:
    struct InFlight {
        cs_prepared* batch;
        size_t first;
    };
    std::deque<InFlight> flight;

    // Appends refilled plans (clay::Renderer::Refill); `wait`: block until some are
    // ready or none remain.
    bool more(bool wait)
    {
        const cs_plan* plans = nullptr;
        size_t count = 0;
        if (!refill || !refill(user, wait ? 1 : 0, &plans, &count) || !count)
            return false;
        checkPlans(plans, count);
        queue.insert(queue.end(), plans, plans + count);
        ++refills;
        return true;
    }

    bool splitGroup(size_t first, size_t jobs) const
    {
        const uint64_t id = queue[first].volume_group;
        const bool continues = first + jobs < queue.size() && id && queue[first + jobs].volume_group == id;
        return r.groupMinimum > 0 && id && (continues || (first > 0 && queue[first - 1].volume_group == id));
    }

    void publishFront()
    {
        InFlight front = flight.front();
        flight.pop_front();
        std::unique_ptr<cs_prepared, void (*)(cs_prepared*)> guard(front.batch, cs_prepared_destroy);
        publishBatch(*front.batch, front.first);
    }

    void drain()
    {
        while (!flight.empty())
            publishFront();
    }

    // Stages `jobs` plans on `lane`; on running out of device memory, first publishes
    // the batches in flight and releases the other lanes' arenas, then halves the
    // batch (src/cuda/renderer.cpp:947-992).  Null when a single job does not fit.
    cs_prepared* tryPrepare(size_t first, size_t& jobs, int lane)
    {
        for (;;) {
            try {
                return prepare(r, queue.data() + first, jobs, true, lane, ticketBase + first);
            } catch (const CudaError& e) {
                if (e.code != cudaErrorMemoryAllocation)
                    throw;
                r.budgetCache = 0;
                bool released = false;
                if (!flight.empty()) {
                    drain();
                    released = true;
                }
                for (int other = 0; other < cs_renderer::kLanes; ++other) {
                    cs_renderer::Lane& l = r.lanes[other];
                    if (other != lane && l.arena) {
                        check(cudaStreamSynchronize(l.stream), "CUDA lane drain");
                        cudaFree(l.arena);
                        r.live -= l.arenaCapacity;
                        l.arena = nullptr;
                        l.arenaCapacity = 0;
                        released = true;
                    }
                }
                if (released)
                    continue;
                if (jobs > 1) {
                    jobs = batchEnd(first, first + jobs / 2) - first;
                    continue;
                }
                // A lone job whose chain scratch dominates: halve the scratch budget,
                // so the job renders in more segments (src/cuda/renderer.cpp:950-953).
                // (The budget only ever shrinks, so the ladder ends.)
                const size_t halved = r.failed.scratch / 2;
                if (r.failed.scratch > std::max<size_t>(r.failed.finishing, size_t(2) << 20) &&
                    (!r.oomBudget || halved < r.oomBudget)) {
                    r.oomBudget = halved;
                    continue;
                }
                size_t freeBytes = 0, total = 0;
                cudaMemGetInfo(&freeBytes, &total);
                std::fprintf(stderr, "MEMORY\tjob=%zu\trequested_bytes=%zu\tmix_bytes=%zu\tfilter_bytes=%zu"
                                     "\tfinishing_bytes=%zu\tmetadata_bytes=%zu\tsample_bytes=%zu"
                                     "\tfree_device_bytes=%zu\n",
                             ticketBase + first, r.failed.requested, r.failed.mix, r.failed.scratch,
                             r.failed.finishing, r.failed.metadata, r.uploaded * sizeof(float), freeBytes);
                return nullptr;
            }
        }
    }

    size_t rejectJob(size_t first)
    {
        rejectScratch(first);
        // A split group whose last member was rejected still publishes the members
        // it retained.
        const uint64_t id = queue[first].volume_group;
        if (!chunks.empty() && !(first + 1 < queue.size() && id && queue[first + 1].volume_group == id))
            finishGroup(nullptr, first);
        return first + 1;
    }

    // One batch with nothing else in flight (chunks of split volume groups), on lane
    // 0; returns the next job.
    size_t renderAlone(size_t first, size_t jobs)
    {
        cs_prepared* prepared = tryPrepare(first, jobs, 0);
        if (!prepared)
            return rejectJob(first);
        std::unique_ptr<cs_prepared, void (*)(cs_prepared*)> guard(prepared, cs_prepared_destroy);
        if (!splitGroup(first, jobs)) {
            run(r, *prepared, nullptr);
            publishBatch(*prepared, first);
        } else {
            const uint64_t id = queue[first].volume_group;
            const bool continues = first + jobs < queue.size() && queue[first + jobs].volume_group == id;
            prepared->deferGroups = true;
            run(r, *prepared, nullptr);
            if (continues)
                retainChunk(*prepared, first);
            else
                finishGroup(prepared, first);
        }
        return first + jobs;
    }

    struct Chunk {
        size_t first = 0;
        std::vector<int> blockJob, jobBlockFirst;
        std::vector<cs_tail_result> results;   // after the chunk's own acceptance layout
        size_t samples = 0;
        void* device = nullptr;                 // waiting on the device
        std::vector<int16_t> host;              // spilled to host memory
        double seconds = 0;
    };

    cs_renderer& r;
    cs_publish_fn publish;
    cs_refill_fn refill;
    void* user;
    std::vector<cs_plan> queue;
    std::vector<Chunk> chunks;                  // the split group rendered so far

    // End of a batch [first, end): stops before a volume group the batch would cut
    // (unless the batch starts with it) and at the end of a split group it continues
    // (trySynthesize's group rule, src/cuda/renderer.cpp:816-829).
    size_t batchEnd(size_t first, size_t end) const
    {
        if (r.groupMinimum <= 0 || end <= first)
            return end;
        const uint64_t head = queue[first].volume_group;
        if (head && first > 0 && queue[first - 1].volume_group == head) {
            size_t stop = first;
            while (stop < end && queue[stop].volume_group == head)
                ++stop;
            return stop;
        }
        if (end < queue.size()) {
            const uint64_t id = queue[end - 1].volume_group;
            if (id && queue[end].volume_group == id) {
                size_t start = end - 1;
                while (start > first && queue[start - 1].volume_group == id)
                    --start;
                if (start > first)
                    return start;
            }
        }
        return end;
    }

    double seconds(cs_prepared& p)
    {
        float ms = 0;
        check(cudaEventElapsedTime(&ms, p.begin, p.end), "CUDA kernel timing");
        return ms / 1000.0;
    }

    void rejectScratch(size_t first)
    {
        cs_batch rejected{};
        rejected.failed_scratch_bytes = std::max<size_t>(r.failed.requested, 1);
        publish(user, &rejected, ticketBase + first);
    }

    void deliver(const int16_t* pcm, size_t samples, const cs_tail_result* results, size_t count, double kernel,
                 size_t first)
    {
        r.downloaded += samples * sizeof(int16_t);
        cs_batch batch{};
        batch.pcm = pcm;
        batch.pcm_samples = samples;
        batch.results = results;
        batch.result_count = count;
        batch.kernel_seconds = kernel;
        publish(user, &batch, ticketBase + first);
    }

    int16_t* hostPcm(size_t samples)
    {
        return static_cast<int16_t*>(cs_renderer::pinned(r.hostPcm, r.hostPcmCapacity,
                                                         std::max<size_t>(samples, 1) * sizeof(int16_t)));
    }

    void publishBatch(cs_prepared& p, size_t first)
    {
        if (p.asyncDownload) {
            check(cudaEventSynchronize(p.copied), "CUDA batch download");
            float copyMs = 0;
            if (cudaEventElapsedTime(&copyMs, p.downloading, p.copied) == cudaSuccess)
                r.hostMs[kPhaseDownload] += copyMs;
            r.hostMs[kPhaseKernels] += 1e3 * seconds(p);
            const auto* buffer = static_cast<const unsigned char*>(r.lanes[p.lane].download);
            int failed = 0;
            std::memcpy(&failed, buffer, sizeof(int));
            if (failed)
                throw std::runtime_error("a device wait ran out of its iteration limit (staged copy did not complete)");
            const auto* results = reinterpret_cast<const cs_tail_result*>(buffer + p.downloadResults);
            const size_t count = p.batch.jobs.size();
            const size_t samples = count ? size_t(results[count - 1].offset + uint64_t(results[count - 1].dataFrames)) *
                (r.natural ? 1 : 2) : 0;
            p.results.assign(results, results + count);
            deliver(reinterpret_cast<const int16_t*>(buffer + p.downloadPcm), samples, p.results.data(), count,
                    seconds(p), first);
            return;
        }
        const size_t samples = collectResults(r, p);
        int16_t* pcm = hostPcm(samples);
        if (samples)
            check(cudaMemcpy(pcm, p.output, samples * sizeof(int16_t), cudaMemcpyDeviceToHost), "CUDA PCM download");
        deliver(pcm, samples, p.results.data(), p.results.size(), seconds(p), first);
    }

    static size_t samplesOf(const std::vector<cs_tail_result>& results, int channels)
    {
        if (results.empty())
            return 0;
        return size_t(results.back().offset + uint64_t(results.back().dataFrames)) * size_t(channels);
    }

    // A chunk that is not the group's last: pack its accepted PCM without gains and
    // keep it (retain, src/cuda/renderer.cpp:1202-1236).
    void retainChunk(cs_prepared& p, size_t first)
    {
        check(cudaStreamSynchronize(r.stream), "CUDA chunk verdicts");
        const int channels = r.natural ? 1 : 2;
        launchPack(p.packView, r.natural, r.stream);
        check(cudaGetLastError(), "CUDA chunk packing launch");
        check(cudaEventRecord(p.end, r.stream), "CUDA timing record");
        collectResults(r, p);
        Chunk chunk;
        chunk.first = first;
        chunk.blockJob = p.batch.blockJob;
        chunk.jobBlockFirst = p.batch.jobBlockFirst;
        chunk.results = p.results;
        chunk.samples = samplesOf(p.results, channels);
        chunk.seconds = seconds(p);
        const size_t bytes = chunk.samples * sizeof(int16_t);
        if (bytes) {
            size_t freeBytes = 0, total = 0;
            check(cudaMemGetInfo(&freeBytes, &total), "CUDA waiting memory budget");
            const size_t limit = std::min(r.waitingLimit, total / 16);
            if (r.waiting <= limit && bytes <= std::min(limit - r.waiting, freeBytes / 4)) {
                if (cudaMalloc(&chunk.device, bytes) == cudaSuccess) {
                    r.waiting += bytes;
                    r.peakWaiting = std::max(r.peakWaiting, r.waiting);
                    r.live += bytes;
                    r.record();
                    check(cudaMemcpy(chunk.device, p.output, bytes, cudaMemcpyDeviceToDevice), "CUDA retain group PCM");
                } else {
                    cudaGetLastError();
                    chunk.device = nullptr;
                }
            }
            if (!chunk.device) {
                chunk.host.resize(chunk.samples);
                check(cudaMemcpy(chunk.host.data(), p.output, bytes, cudaMemcpyDeviceToHost), "CUDA spill group PCM");
                r.spilled += bytes;
            }
        }
        chunks.push_back(std::move(chunk));
    }

    // The group's last chunk: match the whole group's gains, pack and publish this
    // chunk (none when its job was rejected), then pack and publish every retained
    // chunk.
    void finishGroup(cs_prepared* p, size_t first)
    {
        const int channels = r.natural ? 1 : 2;
        std::vector<cs_tail_result> group;
        for (const Chunk& c : chunks)
            group.insert(group.end(), c.results.begin(), c.results.end());
        const size_t local = group.size();
        if (p) {
            collectResults(r, *p);
            group.insert(group.end(), p->results.begin(), p->results.end());
        }
        const size_t resultBytes = std::max<size_t>(group.size(), 1) * sizeof(cs_tail_result);
        void* control = nullptr;
        check(cudaMalloc(&control, resultBytes + sizeof(int2)), "CUDA group control allocation");
        std::unique_ptr<void, cudaError_t (*)(void*)> controlGuard(control, cudaFree);
        auto* results = static_cast<cs_tail_result*>(control);
        auto* range = reinterpret_cast<int2*>(static_cast<unsigned char*>(control) + resultBytes);
        const int2 whole = make_int2(0, int(group.size()));
        if (!group.empty())
            check(cudaMemcpy(results, group.data(), group.size() * sizeof(cs_tail_result), cudaMemcpyHostToDevice),
                  "CUDA group metadata upload");
        check(cudaMemcpy(range, &whole, sizeof whole, cudaMemcpyHostToDevice), "CUDA group upload");
        launchMatch(range, 1, r.groupMinimum, results, r.stream);
        double kernel = 0;
        for (const Chunk& c : chunks)
            kernel += c.seconds;
        if (p) {
            PackView view = p->packView;
            view.results = results + local;
            launchPack(view, r.natural, r.stream);
            check(cudaGetLastError(), "CUDA group packing launch");
            check(cudaStreamSynchronize(r.stream), "CUDA group packing");
            std::vector<cs_tail_result> mine(p->results.size());
            check(cudaMemcpy(mine.data(), view.results, mine.size() * sizeof(cs_tail_result),
                             cudaMemcpyDeviceToHost), "CUDA render metadata download");
            const size_t samples = samplesOf(mine, channels);
            int16_t* pcm = hostPcm(samples);
            if (samples)
                check(cudaMemcpy(pcm, p->output, samples * sizeof(int16_t), cudaMemcpyDeviceToHost),
                      "CUDA PCM download");
            deliver(pcm, samples, mine.data(), mine.size(), kernel + seconds(*p), first);
            kernel = 0;
        } else {
            check(cudaGetLastError(), "CUDA group volume launch");
        }
        size_t at = 0;
        for (Chunk& c : chunks) {
            packRetained(c, results + at, kernel);
            kernel = 0;
            at += c.results.size();
        }
        chunks.clear();
    }

    // packRetained (src/cuda/renderer.cpp:1238-1279): the chunk's waiting PCM with
    // the matched results.
    void packRetained(Chunk& c, cs_tail_result* results, double kernel)
    {
        const int channels = r.natural ? 1 : 2;
        const size_t jobs = c.results.size(), blocks = c.blockJob.size();
        const size_t bytes = c.samples * sizeof(int16_t);
        Layout layout;
        const size_t oBlockJob = layout.add(std::max<size_t>(blocks * sizeof(int), 1));
        const size_t oJobBlock = layout.add(std::max<size_t>(jobs * sizeof(int), 1));
        const size_t oSource = layout.add(std::max<size_t>(jobs * sizeof(uint64_t), 1));
        const size_t oSpill = layout.add(c.device ? 1 : std::max<size_t>(bytes, 1));
        const size_t oOutput = layout.add(std::max<size_t>(bytes, 1));
        void* arena = nullptr;
        check(cudaMalloc(&arena, layout.bytes), "CUDA retained group scratch allocation");
        std::unique_ptr<void, cudaError_t (*)(void*)> arenaGuard(arena, cudaFree);
        auto* base = static_cast<unsigned char*>(arena);
        check(cudaMemcpy(base + oBlockJob, c.blockJob.data(), blocks * sizeof(int), cudaMemcpyHostToDevice),
              "CUDA retained job upload");
        check(cudaMemcpy(base + oJobBlock, c.jobBlockFirst.data(), jobs * sizeof(int), cudaMemcpyHostToDevice),
              "CUDA retained job upload");
        if (!c.device && bytes)
            check(cudaMemcpy(base + oSpill, c.host.data(), bytes, cudaMemcpyHostToDevice), "CUDA spilled PCM upload");
        PackView view{};
        view.blockJob = reinterpret_cast<const int*>(base + oBlockJob);
        view.jobBlockFirst = reinterpret_cast<const int*>(base + oJobBlock);
        view.results = results;
        view.sourceOffset = reinterpret_cast<uint64_t*>(base + oSource);
        view.source = static_cast<const short*>(c.device ? c.device : static_cast<void*>(base + oSpill));
        view.output = reinterpret_cast<short*>(base + oOutput);
        view.jobCount = int(jobs);
        view.blockCount = int(blocks);
        launchPack(view, r.natural, r.stream);
        check(cudaGetLastError(), "CUDA retained packing launch");
        check(cudaStreamSynchronize(r.stream), "CUDA retained packing");
        std::vector<cs_tail_result> packed(jobs);
        check(cudaMemcpy(packed.data(), results, jobs * sizeof(cs_tail_result), cudaMemcpyDeviceToHost),
              "CUDA retained job metadata download");
        const size_t samples = samplesOf(packed, channels);
        int16_t* pcm = hostPcm(samples);
        if (samples)
            check(cudaMemcpy(pcm, view.output, samples * sizeof(int16_t), cudaMemcpyDeviceToHost),
                  "CUDA PCM download");
        if (c.device) {
            cudaFree(c.device);
            c.device = nullptr;
            r.waiting -= bytes;
            r.live -= bytes;
        }
        c.host.clear();
        deliver(pcm, samples, packed.data(), packed.size(), kernel, c.first);
    }
};

} // namespace
} // namespace cs

namespace cs {
namespace {
template <class F>
int guardedOn(cs_renderer* r, F&& body)
{
    const int status = guarded(std::forward<F>(body));
    if (status && r)
        r->error = lastError;
    return status;
}
} // namespace
} // namespace cs

extern "C" {

const char* cs_last_error(void) { return cs::lastError.c_str(); }
const char* cs_renderer_last_error(const cs_renderer* r) { return r ? r->error.c_str() : ""; }

int cs_renderer_create(int device, int natural, const cs_audio_config* audio, int group_minimum,
                       size_t waiting_limit, size_t batch_jobs, cs_renderer** out)
{
    return cs::guarded([&] {
        if (!out)
            throw std::runtime_error("null output handle");
        *out = nullptr;
        auto r = std::make_unique<cs_renderer>();
        r->device = device;
        r->natural = natural != 0;
        if (audio) {
            r->audio = *audio;
        } else {
            r->audio.rate = 44100;
            r->audio.window = 2205;
        }
        if (r->audio.rate <= 0 || r->audio.window <= 0)
            throw std::runtime_error("audio config needs a positive rate and window");
        r->groupMinimum = group_minimum;
        r->waitingLimit = waiting_limit;
        r->batchJobs = std::max<size_t>(1, batch_jobs);
        const int rate = r->audio.rate;
        // TailConfig of the reference renderer (src/cuda/renderer.cpp:492-494).
        r->tail = {r->audio.window, 2 * rate, int(std::nearbyint(rate / 4.)), int(std::nearbyint(rate / 10.)),
                   std::pow(10., -1.5), 32768 * std::pow(10., -3.9), 32768 * std::pow(10., -3.)};
        cs::check(cudaSetDevice(device), "CUDA device");
        cudaDeviceProp prop{};
        cs::check(cudaGetDeviceProperties(&prop, device), "CUDA device properties");
        if (prop.major < 10)
            throw std::runtime_error(std::string("claysampler_b200 needs an sm_100 GPU, found ") + prop.name);
        r->name = prop.name;
        int leastPriority = 0, greatestPriority = 0;
        cs::check(cudaDeviceGetStreamPriorityRange(&leastPriority, &greatestPriority), "CUDA stream priorities");
        cs::check(cudaStreamCreateWithFlags(&r->compute, cudaStreamNonBlocking), "CUDA stream");
        for (auto& lane : r->lanes) {
            cs::check(cudaStreamCreateWithFlags(&lane.stream, cudaStreamNonBlocking), "CUDA stream");
            cs::check(cudaEventCreateWithFlags(&lane.staged, cudaEventDisableTiming), "CUDA event");
            cs::check(cudaEventCreateWithFlags(&lane.computed, cudaEventDisableTiming), "CUDA event");
            for (int k = 0; k < cs::kLeadTiers; ++k) {
                cs::check(cudaStreamCreateWithPriority(&lane.lead[k], cudaStreamNonBlocking, greatestPriority),
                          "CUDA stream");
                cs::check(cudaEventCreateWithFlags(&lane.leadReady[k], cudaEventDisableTiming), "CUDA event");
                cs::check(cudaEventCreateWithFlags(&lane.leadDone[k], cudaEventDisableTiming), "CUDA event");
            }
        }
        r->stream = r->lanes[0].stream;
        std::vector<float> table(size_t(cs::kTaps) * (cs::kPhases + 1));
        cs::buildSincTable(table.data());
        cs::check(cudaMalloc(&r->sinc, table.size() * sizeof(float)), "CUDA sinc table");
        cs::check(cudaMemcpy(r->sinc, table.data(), table.size() * sizeof(float), cudaMemcpyHostToDevice),
                  "CUDA sinc upload");
        size_t freeBytes = 0, total = 0;
        cs::check(cudaMemGetInfo(&freeBytes, &total), "CUDA sample cache budget");
        r->cacheBudget = std::min(freeBytes - freeBytes / 3, total / 2);
        r->record();
        *out = r.release();
    });
}

void cs_renderer_destroy(cs_renderer* r)
{
    if (!r)
        return;
    r->service.reset();
    cudaSetDevice(r->device);
    for (auto& lane : r->lanes)
        if (lane.stream) cudaStreamSynchronize(lane.stream);
    if (r->compute) cudaStreamSynchronize(r->compute);
    cudaFree(r->sinc);
    cudaFree(r->bank);
    cudaFree(r->windowPool);
    for (auto& lane : r->lanes) {
        for (cudaStream_t lead : lane.lead)
            if (lead) cudaStreamSynchronize(lead);
        cudaFree(lane.arena);
    }
    if (r->hostPcm) cudaFreeHost(r->hostPcm);
    if (r->staging) cudaFreeHost(r->staging);
    for (auto& lane : r->lanes) {
        if (lane.download) cudaFreeHost(lane.download);
        if (lane.staging) cudaFreeHost(lane.staging);
        if (lane.uploaded) cudaEventDestroy(lane.uploaded);
        if (lane.staged) cudaEventDestroy(lane.staged);
        if (lane.computed) cudaEventDestroy(lane.computed);
    }
    if (r->compute) cudaStreamDestroy(r->compute);
    for (auto& lane : r->lanes) {
        if (lane.stream) cudaStreamDestroy(lane.stream);
        for (int k = 0; k < cs::kLeadTiers; ++k) {
            if (lane.lead[k]) cudaStreamDestroy(lane.lead[k]);
            if (lane.leadReady[k]) cudaEventDestroy(lane.leadReady[k]);
            if (lane.leadDone[k]) cudaEventDestroy(lane.leadDone[k]);
        }
    }
    delete r;
}

int cs_upload_samples(cs_renderer* r, const float* pcm, size_t floats, int fresh)
{
    return cs::guardedOn(r, [&] {
        if (!r)
            throw std::runtime_error("null renderer");
        cs::check(cudaSetDevice(r->device), "CUDA device");
        r->budgetCache = 0;
        if (fresh)
            r->uploaded = 0;
        if (floats <= r->uploaded && r->bank)
            return;
        if (floats > r->bankCapacity) {
            // Grow with slack and keep what was uploaded (src/cuda/renderer.cpp:564-586).
            const size_t capacity = floats + std::min(floats / 2, size_t(32) << 20);
            float* grown = nullptr;
            cs::check(cudaMalloc(&grown, capacity * sizeof(float)), "CUDA sample bank allocation");
            if (r->uploaded)
                cs::check(cudaMemcpy(grown, r->bank, r->uploaded * sizeof(float), cudaMemcpyDeviceToDevice),
                          "CUDA sample bank growth");
            cudaFree(r->bank);
            r->bank = grown;
            r->bankCapacity = capacity;
        }
        if (floats > r->uploaded)
            cs::check(cudaMemcpy(r->bank + r->uploaded, pcm + r->uploaded, (floats - r->uploaded) * sizeof(float),
                                 cudaMemcpyHostToDevice), "CUDA sample upload");
        r->uploaded = floats;
        r->record();
    });
}

int cs_prepare(cs_renderer* r, const cs_plan* plans, size_t count, cs_prepared** out)
{
    return cs::guardedOn(r, [&] {
        if (!r || !out)
            throw std::runtime_error("null renderer or output handle");
        cs::checkPlans(plans, count);
        *out = cs::prepare(*r, plans, count);
    });
}

int cs_run(cs_renderer* r, cs_prepared* p, void* stream)
{
    return cs::guardedOn(r, [&] {
        if (!r || !p)
            throw std::runtime_error("null renderer or batch");
        if (!r->bank && !p->batch.voices.empty())
            throw std::runtime_error("no sample bank uploaded");
        cs::run(*r, *p, static_cast<cudaStream_t>(stream));
    });
}

int cs_collect(cs_renderer* r, cs_prepared* p, int16_t* pcm, size_t capacity, size_t* samples,
               cs_tail_result* results)
{
    return cs::guardedOn(r, [&] {
        if (!r || !p || !p->ran)
            throw std::runtime_error("batch has not been run");
        const size_t count = cs::collectResults(*r, *p);
        if (samples)
            *samples = count;
        if (results && !p->results.empty())
            std::memcpy(results, p->results.data(), p->results.size() * sizeof(cs_tail_result));
        if (pcm) {
            if (capacity < count)
                throw std::runtime_error("PCM buffer too small");
            if (count)
                cs::check(cudaMemcpy(pcm, p->output, count * sizeof(int16_t), cudaMemcpyDeviceToHost),
                          "CUDA PCM download");
            r->downloaded += count * sizeof(int16_t);
        }
    });
}

int cs_copy_mix(cs_renderer* r, cs_prepared* p, void* host, size_t bytes)
{
    return cs::guardedOn(r, [&] {
        if (!r || !p || !p->ran)
            throw std::runtime_error("batch has not been run");
        if (bytes < p->mixBytes)
            throw std::runtime_error("mix buffer too small");
        cs::check(cudaEventSynchronize(p->end), "CUDA render completion");
        cs::check(cudaMemcpy(host, p->view.mix, p->mixBytes, cudaMemcpyDeviceToHost), "CUDA mix download");
    });
}

size_t cs_prepared_frames(const cs_prepared* p) { return p ? p->batch.frames : 0; }

int cs_prepared_mix_device(const cs_prepared* p, const void** mix, size_t* bytes)
{
    return cs::guarded([&] {
        if (!p || !mix || !bytes)
            throw std::runtime_error("null argument");
        *mix = p->view.mix;
        *bytes = p->mixBytes;
    });
}

int cs_prepared_set_profile(cs_prepared* p, int enable)
{
    return cs::guarded([&] {
        if (!p)
            throw std::runtime_error("null batch");
        p->profile = enable != 0;
    });
}

int cs_prepared_stage_ms(cs_prepared* p, float* ms, int capacity)
{
    int stages = 0;
    const int status = cs::guarded([&] {
        if (!p || !p->ran || !p->profile)
            throw std::runtime_error("batch has no profiled run");
        cs::check(cudaEventSynchronize(p->end), "CUDA render completion");
        for (int i = 0; i < capacity; ++i)
            ms[i] = 0;
        for (size_t k = 1; k < p->markStage.size(); ++k) {
            float elapsed = 0;
            cs::check(cudaEventElapsedTime(&elapsed, p->marks[k - 1], p->marks[k]), "CUDA stage timing");
            const int id = p->markStage[k];
            if (id >= 0 && id < capacity)
                ms[id] += elapsed;
        }
        stages = cs::kStages;
    });
    return status ? -1 : stages;
}

const char* cs_stage_name(int stage) { return stage >= 0 && stage < cs::kStages ? cs::kStageNames[stage] : ""; }
int cs_prepared_launches(const cs_prepared* p) { return p ? p->launches : 0; }

void cs_prepared_destroy(cs_prepared* p)
{
    if (!p)
        return;
    if (p->end) cudaEventSynchronize(p->end);
    for (cudaEvent_t e : p->marks)
        cudaEventDestroy(e);
    if (p->copied) cudaEventSynchronize(p->copied);
    if (p->begin) cudaEventDestroy(p->begin);
    if (p->end) cudaEventDestroy(p->end);
    if (p->copied) cudaEventDestroy(p->copied);
    if (p->downloading) cudaEventDestroy(p->downloading);
    if (p->arena && !p->sharedArena) {
        cudaFree(p->arena);
        if (p->owner)
            p->owner->live -= p->arenaBytes;
    }
    delete p;
}

int cs_render_window(cs_renderer* r, const cs_plan* plans, size_t count, cs_publish_fn publish,
                     cs_refill_fn refill, void* user)
{
    return cs::guardedOn(r, [&] {
        if (!r || !publish)
            throw std::runtime_error("null renderer or publish callback");
        cs::checkPlans(plans, count);
        if (r->service && (r->service->pending() || r->service->inFlight()))
            throw std::runtime_error("submitted jobs are still being rendered: poll them first");
        cs::WindowRenderer(*r, publish, refill, user).render(plans, count);
    });
}

int cs_submit(cs_renderer* r, const cs_plan* plans, size_t count, uint64_t* first_ticket)
{
    return cs::guardedOn(r, [&] {
        if (!r)
            throw std::runtime_error("null renderer");
        cs::checkPlans(plans, count);
        if (!r->service)
            r->service = std::make_unique<cs::WindowRenderer>(*r, nullptr, nullptr, nullptr);
        const size_t ticket = r->service->submit(plans, count);
        if (first_ticket)
            *first_ticket = ticket;
    });
}

int cs_poll(cs_renderer* r, int wait, cs_publish_fn publish, void* user, size_t* published)
{
    return cs::guardedOn(r, [&] {
        if (!r || !publish)
            throw std::runtime_error("null renderer or publish callback");
        const size_t count = r->service ? r->service->poll(wait != 0, publish, user) : 0;
        if (published)
            *published = count;
    });
}

size_t cs_pending_jobs(const cs_renderer* r)
{
    if (!r || !r->service)
        return 0;
    size_t jobs = r->service->pending();
    return jobs + r->service->inFlightJobs();
}

const char* cs_renderer_device(const cs_renderer* r) { return r ? r->name.c_str() : ""; }
size_t cs_peak_bytes(const cs_renderer* r) { return r ? r->peak : 0; }
size_t cs_sample_cache_budget(const cs_renderer* r) { return r ? r->cacheBudget : 0; }
size_t cs_peak_waiting_bytes(const cs_renderer* r) { return r ? r->peakWaiting : 0; }
size_t cs_spilled_bytes(const cs_renderer* r) { return r ? r->spilled : 0; }
size_t cs_downloaded_bytes(const cs_renderer* r) { return r ? r->downloaded : 0; }

// Caps the chain-storage bytes of one synthesis segment (0 restores the default
// derived from free device memory).  No reference counterpart: the reference
// exercises segmentation with a special build that limits scratch to 64 KiB.
int cs_renderer_set_scratch_limit(cs_renderer* r, size_t bytes)
{
    return cs::guardedOn(r, [&] {
        if (!r)
            throw std::runtime_error("null renderer");
        r->scratchLimit = bytes;
    });
}

int cs_renderer_fail_allocations(cs_renderer* r, int count)
{
    return cs::guardedOn(r, [&] {
        if (!r || count < 0)
            throw std::runtime_error("invalid allocation-failure count");
        r->failAllocations = count;
    });
}

int cs_renderer_set_ordered_compute(cs_renderer* r, int ordered)
{
    return cs::guardedOn(r, [&] {
        if (!r)
            throw std::runtime_error("null renderer");
        if (r->service && (r->service->pending() || r->service->inFlight()))
            throw std::runtime_error("submitted jobs are in flight; poll them first");
        r->orderedCompute = ordered != 0;
    });
}

int cs_renderer_set_lanes(cs_renderer* r, int lanes)
{
    return cs::guardedOn(r, [&] {
        if (!r)
            throw std::runtime_error("null renderer");
        if (lanes < 1 || lanes > cs_renderer::kLanes)
            throw std::runtime_error("lanes must be 1 to " + std::to_string(cs_renderer::kLanes));
        r->laneCount = lanes;
    });
}

size_t cs_renderer_deferred_launches(const cs_renderer* r) { return r ? r->deferred : 0; }

int cs_renderer_host_ms(const cs_renderer* r, double* ms, int capacity)
{
    if (!r || !ms)
        return 0;
    for (int i = 0; i < capacity && i < cs::kHostPhases; ++i)
        ms[i] = r->hostMs[i];
    return cs::kHostPhases;
}

int cs_renderer_set_shared_sources(cs_renderer* r, int enable)
{
    return cs::guardedOn(r, [&] {
        if (!r)
            throw std::runtime_error("null renderer");
        r->sharedSources = enable != 0;
    });
}

size_t cs_prepared_shared_sources(const cs_prepared* p) { return p ? p->shared.sources.size() : 0; }
size_t cs_prepared_shared_frames(const cs_prepared* p) { return p ? p->shared.floats : 0; }
long long cs_prepared_shared_voice_frames(const cs_prepared* p) { return p ? p->shared.sharedVoiceFrames : 0; }
long long cs_prepared_shared_sinc(const cs_prepared* p, long long* voice_floats)
{
    if (voice_floats)
        *voice_floats = p ? p->shared.sincVoiceFloats : 0;
    return p ? p->shared.sincFloats : 0;
}

size_t cs_prepared_segments(const cs_prepared* p) { return p ? p->tables.segments.size() : 0; }

} // extern "C"
